// 3x3x3 convolution as an implicit GEMM on the 5th-generation tensor cores
// (tcgen05, sm_100a), used by the learned torso preconditioner.
//
// Tensors are BF16, channels innermost: X[D][H][W][CIN], Y[D][H][W][COUT];
// W must be a multiple of 128 and CIN, COUT multiples of 16.  One CTA
// computes one output line tile: 128 consecutive voxels along W at fixed
// (d, h), all COUT channels:
//   GEMM  M = 128 voxels, N = COUT, K = 27 taps x CIN
// accumulated in FP32 in tensor memory (TMEM, 128 lanes x COUT columns).
//
// The K loop runs over the 9 (dz, dy) input lines.  For each line a TMA
// load brings the 130 voxels w0-1 .. w0+128 (zero-filled outside the grid)
// into shared memory as CIN/8 chunks of [130 voxels][8 channels] -- exactly
// the no-swizzle K-major core-matrix layout of the UMMA A operand (8 rows of
// 16 bytes per core matrix, 8-row groups 128 B apart, channel groups one
// chunk apart).  The three dx taps of the line are the same smem tile with
// the descriptor start moved by +/-16 bytes (one voxel row), so each line is
// loaded once and used three times.  The weights of the three taps of the
// line ([tap][CIN/8][COUT][8], K-major B operand) arrive by one bulk copy.
// Two smem stages alternate; a single thread issues the TMA copies and the
// MMAs and commits each stage's MMAs to that stage's "empty" barrier.
//
// Every mbarrier wait is bounded: on timeout the CTA records the location in
// *err, stops issuing work, waits (bounded) for its own copies, frees its
// TMEM and returns; the host reads *err after the launch.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/hrdaya_b200.h"

namespace hp {
namespace tc {

constexpr int TILE_M = 128;           // voxels per CTA (GEMM M)
constexpr int LINE = 130;             // voxels loaded per line (tile + halo)
constexpr int CHUNK = 2176;           // bytes per 8-channel chunk (130*16 rounded up to 128 B)
constexpr uint32_t SPIN_LIMIT = 1u << 26;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// Bounded wait for the phase with parity `parity` to complete.  Returns
// false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (uint32_t it = 0; it < SPIN_LIMIT; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Bounded wait that also gives up once another role of the CTA has set
// *failed (checked every 256 polls).  Returns false on timeout or failure.
__device__ __forceinline__ bool mbar_wait_f(uint64_t* bar, uint32_t parity,
                                            const volatile int* failed) {
  const uint32_t a = smem_u32(bar);
  for (uint32_t it = 0; it < SPIN_LIMIT; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if ((it & 255u) == 255u && *failed) return false;
  }
  return false;
}

// The same for waiters that are not on the critical path (epilogue warps
// waiting for a finished accumulator): a short sleep between polls keeps
// them from taking issue slots from the copy and MMA threads.  Bounded at
// about 2^22 polls (about a second).
__device__ __forceinline__ bool mbar_wait_sleep(uint64_t* bar, uint32_t parity,
                                                const volatile int* failed) {
  const uint32_t a = smem_u32(bar);
  for (uint32_t it = 0; it < (1u << 22); ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (*failed) return false;
    __nanosleep(200);
  }
  return false;
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 4-D tiled TMA load (no multicast), completion on `bar`.
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1,
                                            int c2, int c3, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
      "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}

// Untiled bulk copy global -> shared (16-byte aligned, size multiple of 16).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes,
                                          uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"((uint64_t)src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// UMMA shared-memory descriptor, no swizzle, K-major: rows of 16 bytes,
// 8-row groups `sbo` bytes apart, the two 8-element K chunks `lbo` bytes
// apart (bit layout of the sm100 smem descriptor: start>>4 [0,14),
// LBO>>4 [16,30), SBO>>4 [32,46), version 1 [46,48), layout 0 [61,64)).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm100
  return d;
}

// The descriptor of the same layout at saddr + off: the start field holds
// (address >> 4) in 14 bits and shared-memory addresses stay below 2^18, so
// adding (off >> 4) never carries into the stride fields.  Lets an MMA loop
// build each operand's descriptor once per stage.
__device__ __forceinline__ uint64_t desc_add(uint64_t desc, uint32_t off) {
  return desc + (uint64_t)(off >> 4);
}

// Instruction descriptor, kind::f16: BF16 x BF16 -> FP32, both K-major.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4)                       // D format F32
         | (1u << 7)                     // A format BF16
         | (1u << 10)                    // B format BF16
         | ((uint32_t)(N >> 3) << 17)    // N / 8
         | ((uint32_t)(M >> 4) << 24);   // M / 16
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(dst_smem)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

enum Epi : int {
  EPI_RELU = 0,     // y = relu(acc + bias)                 (bf16)
  EPI_LINEAR = 1,   // y = acc + bias                        (bf16)
  EPI_MASK = 2,     // y = acc * (mask > 0)                  (bf16)  ReLU backward
  EPI_F32_C0 = 3    // y = acc[:, 0] + bias[0]               (fp32, one channel)
};

// Host launcher of the convolution (conv.cu): epi 0 relu(acc + b),
// 1 acc + b, 2 acc * (mask > 0), 3 fp32 channel 0.
hp_status conv3_launch(const void* X, const void* Wp, const float* bias, void* Y,
                       const void* mask, int D, int H, int W, int cin, int cout, int epi,
                       int* err, cudaStream_t s);

// Weight gradient of one layer (conv.cu): gw [cout][cin][27] and gb [cout]
// (FP32, overwritten) from X [D][H][W][cin] and G [D][H][W][max(cout, 16)]
// (bf16), partial sums in `work` (wgrad3_workspace bytes).
int64_t wgrad3_workspace(int D, int H, int W, int cin, int cout);
hp_status wgrad3_launch(const void* X, const void* G, int D, int H, int W, int cin, int cout,
                        float* gw, float* gb, void* work, int64_t work_bytes, int* err,
                        cudaStream_t s);

template <int N>
struct TmemCols {
  static constexpr uint32_t value = N <= 32 ? 32 : (N <= 64 ? 64 : (N <= 128 ? 128 : 256));
};

}  // namespace tc
}  // namespace hp
