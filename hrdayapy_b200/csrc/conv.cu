// tcgen05 3x3x3 convolution kernels (see tc_conv.cuh for the design) and
// their C entry points.
#include "hp_common.cuh"
#include "tc_conv.cuh"

#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>

namespace hp {
namespace tc {

template <int CIN, int COUT>
struct ConvCfg {
  static constexpr int G = CIN / 8;
  static constexpr int A_BYTES = G * CHUNK;
  static constexpr int A_TX = G * LINE * 16;
  static constexpr int B_BYTES = 3 * CIN * COUT * 2;
  static constexpr int STAGE = A_BYTES + B_BYTES;
  static constexpr int SMEM = 2 * STAGE + 128;
  static constexpr uint32_t COLS = TmemCols<COUT>::value;
  static constexpr uint32_t IDESC = idesc_bf16(TILE_M, COUT);
  static_assert(CIN % 16 == 0 && COUT % 16 == 0 && COUT <= 256, "channel counts");
  static_assert(B_BYTES % 128 == 0, "stage alignment");
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(128)
conv3_tc_kernel(const __grid_constant__ CUtensorMap tmX, const __nv_bfloat16* __restrict__ Wp,
                const float* __restrict__ bias, void* __restrict__ Yv,
                const __nv_bfloat16* __restrict__ mask, int D, int H, int W, int epi, int* err) {
  using C = ConvCfg<CIN, COUT>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
  __shared__ __align__(8) uint64_t full[2];
  __shared__ __align__(8) uint64_t empty[2];
  __shared__ __align__(8) uint64_t done;
  __shared__ uint32_t tmem_base;
  __shared__ int failed;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int w0 = blockIdx.x * TILE_M, h = blockIdx.y, d = blockIdx.z;

  if (tid == 0) {
    mbar_init(&full[0], 1);
    mbar_init(&full[1], 1);
    mbar_init(&empty[0], 1);
    mbar_init(&empty[1], 1);
    mbar_init(&done, 1);
    failed = 0;
    fence_barrier_init();
  }
  if (warp == 0) tmem_alloc(&tmem_base, C::COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base;

  if (tid == 0) {
    auto issue = [&](int s, int buf) {
      const int dz = s / 3 - 1, dy = s % 3 - 1;
      uint8_t* A = smem + buf * C::STAGE;
      uint8_t* B = A + C::A_BYTES;
      mbar_expect_tx(&full[buf], C::A_TX + C::B_BYTES);
#pragma unroll
      for (int g = 0; g < C::G; ++g)
        tma_load_4d(A + g * CHUNK, &tmX, g * 8, w0 - 1, h + dy, d + dz, &full[buf]);
      const int tap0 = 9 * (dz + 1) + 3 * (dy + 1);
      bulk_load(B, Wp + (size_t)tap0 * CIN * COUT, C::B_BYTES, &full[buf]);
    };
    int issued = 0;
    issue(0, 0);
    issue(1, 1);
    issued = 2;
    int consumed = 0;
    for (int s = 0; s < 9; ++s) {
      const int buf = s & 1;
      const uint32_t par = (s >> 1) & 1;
      if (!mbar_wait(&full[buf], par)) {
        atomicOr(err, 1);
        failed = 1;
        break;
      }
      tc_fence_after();
      const uint32_t a0 = smem_u32(smem + buf * C::STAGE);
      const uint64_t a_d = smem_desc(a0, CHUNK, 128);
      const uint64_t b_d = smem_desc(a0 + C::A_BYTES, COUT * 16, 128);
#pragma unroll
      for (int dx = 0; dx < 3; ++dx) {
#pragma unroll
        for (int k = 0; k < CIN / 16; ++k) {
          const uint64_t ad = desc_add(a_d, 2 * k * CHUNK + dx * 16);
          const uint64_t bd = desc_add(b_d, (dx * C::G + 2 * k) * COUT * 16);
          mma_bf16(tmem, ad, bd, C::IDESC, (s | dx | k) != 0);
        }
      }
      mma_commit(&empty[buf]);
      consumed = s + 1;
      if (s + 2 < 9) {
        if (!mbar_wait(&empty[buf], par)) {
          atomicOr(err, 2);
          failed = 1;
          break;
        }
        issue(s + 2, buf);
        ++issued;
      }
    }
    if (failed) {
      // let the copies already issued land before the CTA releases smem
      for (int s = consumed; s < issued; ++s) (void)mbar_wait(&full[s & 1], (s >> 1) & 1);
    }
    mma_commit(&done);
  }
  __syncthreads();
  const bool ok = mbar_wait(&done, 0) && !failed;
  if (!ok && tid == 0) atomicOr(err, 4);
  tc_fence_after();
  if (ok) {
    // epilogue: this thread owns output voxel w0 + tid, TMEM lane tid
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
    const int64_t vox = ((int64_t)d * H + h) * W + w0 + tid;
    if (epi == EPI_F32_C0) {
      float v[16];
      tmem_ld16(trow, v);
      ((float*)Yv)[vox] = v[0] + bias[0];
    } else {
      __nv_bfloat16* Y = (__nv_bfloat16*)Yv;
#pragma unroll
      for (int c0 = 0; c0 < COUT; c0 += 16) {
        float v[16];
        tmem_ld16(trow + c0, v);
        __align__(16) __nv_bfloat16 o[16];
        if (epi == EPI_MASK) {
          const uint4* mp = (const uint4*)(mask + vox * COUT + c0);
          __align__(16) __nv_bfloat16 m[16];
          *(uint4*)&m[0] = mp[0];
          *(uint4*)&m[8] = mp[1];
#pragma unroll
          for (int q = 0; q < 16; ++q)
            o[q] = __float2bfloat16(__bfloat162float(m[q]) > 0.0f ? v[q] : 0.0f);
        } else {
#pragma unroll
          for (int q = 0; q < 16; ++q) {
            float y = v[q] + bias[c0 + q];
            if (epi == EPI_RELU) y = fmaxf(y, 0.0f);
            o[q] = __float2bfloat16(y);
          }
        }
        uint4* yp = (uint4*)(Y + vox * COUT + c0);
        yp[0] = *(uint4*)&o[0];
        yp[1] = *(uint4*)&o[8];
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, C::COLS);
}

// -------------------------------------------------------------------------
// Row-blocked variant: one CTA computes R output lines (h0 .. h0+R-1 at the
// same (d, w0..w0+127)), one TMEM accumulator of COUT FP32 columns per line.
// One thread issues the copies up to NS stages ahead, another the products
// (copy latency no longer serialises with the products' completion).
// The K loop runs over dz and the R+2 input lines h0-1 .. h0+R of that
// depth slice: each input line is loaded once and feeds every output line
// within one row of it (up to three), and the 9 (dy, dx) taps of a depth
// slice arrive in one bulk copy per slice -- against one line tile per CTA,
// which loads every input line three times per depth slice and the weights
// nine times.  Two weight buffers (slice zi uses buffer zi & 1; a buffer is
// rewritten only after the MMAs of every stage that read it have completed,
// which the line-stage "empty" wait already guarantees because stages
// complete in order).
template <int CIN, int COUT, int R>
struct RowsCfg {
  static constexpr int G = CIN / 8;
  static constexpr int A_BYTES = G * CHUNK;
  static constexpr int A_TX = G * LINE * 16;
  static constexpr int B_BYTES = 9 * CIN * COUT * 2;
  static constexpr int ACC = (COUT + 31) / 32 * 32;   // TMEM columns per output line
  static constexpr uint32_t COLS = R * ACC <= 32 ? 32 : (R * ACC <= 64 ? 64 : (R * ACC <= 128 ? 128 : (R * ACC <= 256 ? 256 : 512)));
  // line stages in flight: four where that keeps the CTA's shared memory
  // small (48 KB), else two (more CTAs per SM measured faster there)
  static constexpr int NS = 4 * A_BYTES + 2 * B_BYTES + 128 <= 48 * 1024 ? 4 : 2;
  static constexpr int SMEM = NS * A_BYTES + 2 * B_BYTES + 128;
  static constexpr int NSTG = 3 * (R + 2);
  static constexpr uint32_t IDESC = idesc_bf16(TILE_M, COUT);
  static_assert(CIN % 16 == 0 && COUT % 16 == 0 && COUT <= 256, "channel counts");
  static_assert(R * ACC <= 512, "TMEM columns");
  static_assert(B_BYTES % 128 == 0 && A_BYTES % 128 == 0, "stage alignment");
};

constexpr int CONV_ROWS = 4;

template <int CIN, int COUT, int R>
__global__ void __launch_bounds__(128)
conv3_tc_rows_kernel(const __grid_constant__ CUtensorMap tmX, const __nv_bfloat16* __restrict__ Wp,
                     const float* __restrict__ bias, void* __restrict__ Yv,
                     const __nv_bfloat16* __restrict__ mask, int D, int H, int W, int epi,
                     int* err) {
  using C = RowsCfg<CIN, COUT, R>;
  constexpr int NS = C::NS;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
  __shared__ __align__(8) uint64_t full[NS];
  __shared__ __align__(8) uint64_t empty[NS];
  __shared__ __align__(8) uint64_t done;
  __shared__ uint32_t tmem_base;
  __shared__ volatile int failed;
  __shared__ int issued_s, consumed_s;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int w0 = blockIdx.x * TILE_M, h0 = blockIdx.y * R, d = blockIdx.z;

  if (tid == 0) {
    for (int b = 0; b < NS; ++b) {
      mbar_init(&full[b], 1);
      mbar_init(&empty[b], 1);
    }
    mbar_init(&done, 1);
    failed = 0;
    issued_s = 0;
    consumed_s = 0;
    fence_barrier_init();
  }
  if (warp == 0) tmem_alloc(&tmem_base, C::COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base;
  uint8_t* const Bbase = smem + NS * C::A_BYTES;

  // Producer (thread 32): line stage s goes to buffer s % NS; it is
  // refilled once the products of the stage that last used it completed
  // (its "empty" barrier), so the copies run up to NS stages ahead of the
  // products.  A weight buffer is rewritten (first stage of slice 2) only
  // after the products of every stage of slice 0 completed: stages complete
  // in order and slice 0 ends at least NS stages earlier.
  if (tid == 32) {
    int s = 0;
    for (; s < C::NSTG && !failed; ++s) {
      const int buf = s % NS;
      if (s >= NS && !mbar_wait(&empty[buf], ((s / NS) - 1) & 1)) {
        atomicOr(err, 2);
        failed = 1;
        break;
      }
      const int zi = s / (R + 2), ri = s % (R + 2);
      uint8_t* A = smem + buf * C::A_BYTES;
      const bool new_slice = ri == 0;
      mbar_expect_tx(&full[buf], C::A_TX + (new_slice ? C::B_BYTES : 0));
#pragma unroll
      for (int g = 0; g < C::G; ++g)
        tma_load_4d(A + g * CHUNK, &tmX, g * 8, w0 - 1, h0 - 1 + ri, d + zi - 1, &full[buf]);
      if (new_slice)
        bulk_load(Bbase + (zi & 1) * C::B_BYTES, Wp + (size_t)9 * zi * CIN * COUT, C::B_BYTES,
                  &full[buf]);
    }
    issued_s = s;
  }
  // MMA issuer (thread 0)
  if (tid == 0) {
    int s = 0;
    for (; s < C::NSTG; ++s) {
      const int buf = s % NS;
      if (failed || !mbar_wait(&full[buf], (s / NS) & 1)) {
        atomicOr(err, 1);
        failed = 1;
        break;
      }
      tc_fence_after();
      const int zi = s / (R + 2), ri = s % (R + 2);
      const uint64_t a_d = smem_desc(smem_u32(smem + buf * C::A_BYTES), CHUNK, 128);
      const uint64_t b_d = smem_desc(smem_u32(Bbase + (zi & 1) * C::B_BYTES), COUT * 16, 128);
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int dy = ri - 1 - r;   // input line h0-1+ri feeds output line h0+r
        if (dy < -1 || dy > 1) continue;
        const uint32_t td = tmem + (uint32_t)(r * C::ACC);
#pragma unroll
        for (int dx = 0; dx < 3; ++dx) {
#pragma unroll
          for (int k = 0; k < CIN / 16; ++k) {
            const uint64_t ad = desc_add(a_d, 2 * k * CHUNK + dx * 16);
            const uint64_t bd =
                desc_add(b_d, ((3 * (dy + 1) + dx) * C::G + 2 * k) * COUT * 16);
            // the first product into line r (zi 0, dy -1, dx 0, k 0) overwrites
            const uint32_t acc = (zi != 0 || dy != -1 || dx != 0 || k != 0) ? 1u : 0u;
            mma_bf16(td, ad, bd, C::IDESC, acc);
          }
        }
      }
      mma_commit(&empty[buf]);
    }
    consumed_s = s;
    mma_commit(&done);
  }
  __syncthreads();
  if (tid == 32 && failed) {
    // let the copies already issued land before the CTA releases smem
    for (int s = consumed_s; s < issued_s; ++s) (void)mbar_wait(&full[s % NS], (s / NS) & 1);
  }
  __syncthreads();
  const bool ok = mbar_wait(&done, 0) && !failed;
  if (!ok && tid == 0) atomicOr(err, 4);
  tc_fence_after();
  if (ok) {
    // epilogue: this thread owns voxel w0 + tid of every output line, TMEM lane tid
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
    for (int r = 0; r < R; ++r) {
      if (h0 + r >= H) break;
      const uint32_t tl = trow + (uint32_t)(r * C::ACC);
      const int64_t vox = ((int64_t)d * H + h0 + r) * W + w0 + tid;
      if (epi == EPI_F32_C0) {
        float v[16];
        tmem_ld16(tl, v);
        ((float*)Yv)[vox] = v[0] + bias[0];
      } else {
        __nv_bfloat16* Y = (__nv_bfloat16*)Yv;
#pragma unroll
        for (int c0 = 0; c0 < COUT; c0 += 16) {
          float v[16];
          tmem_ld16(tl + c0, v);
          __align__(16) __nv_bfloat16 o[16];
          if (epi == EPI_MASK) {
            const uint4* mp = (const uint4*)(mask + vox * COUT + c0);
            __align__(16) __nv_bfloat16 m[16];
            *(uint4*)&m[0] = mp[0];
            *(uint4*)&m[8] = mp[1];
#pragma unroll
            for (int q = 0; q < 16; ++q)
              o[q] = __float2bfloat16(__bfloat162float(m[q]) > 0.0f ? v[q] : 0.0f);
          } else {
#pragma unroll
            for (int q = 0; q < 16; ++q) {
              float y = v[q] + bias[c0 + q];
              if (epi == EPI_RELU) y = fmaxf(y, 0.0f);
              o[q] = __float2bfloat16(y);
            }
          }
          uint4* yp = (uint4*)(Y + vox * COUT + c0);
          yp[0] = *(uint4*)&o[0];
          yp[1] = *(uint4*)&o[8];
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, C::COLS);
}

// -------------------------------------------------------------------------
// Persistent warp-specialised variant.  One CTA per SM walks the tiles
// (128 voxels along W x R output lines x one depth) t = blockIdx.x,
// blockIdx.x + gridDim.x, ... with three roles:
//   warp 0, lane 0: producer -- the line stages of every tile in one
//     continuous sequence (dz-major, R + 2 input lines per depth slice,
//     TMA line loads plus the slice's 9-tap weight block on the slice's
//     first line) into an NS-stage ring, refilling a stage once the
//     products that read it completed;
//   warp 1, lane 0: MMA issuer -- the products of tile j into one of two
//     TMEM accumulator sets (R lines x ACC columns each, set j & 1), then a
//     commit that hands the set to the epilogue;
//   warps 2-5: epilogue -- each thread owns TMEM lane (warp & 3) * 32 +
//     lane, i.e. one voxel of the tile: it reads the R lines' accumulators,
//     applies the epilogue, stores, and releases the set, while the products
//     of the next tile run in the other set.
// The weight block of a depth slice is double-buffered by global slice
// index; a buffer is rewritten at the first stage of the slice two later,
// whose ring wait (NS <= R + 2 stages back) already covers every product of
// the slice that read it.  Every wait is bounded; on a timeout the role
// records the location in *err and sets a shared flag that makes the other
// roles stop, the CTA waits (bounded) for its copies and products in
// flight, frees its TMEM and returns.
template <int CIN, int COUT, int RR>
struct PersistCfg {
  static constexpr int G = CIN / 8;
  static constexpr int A_BYTES = G * CHUNK;
  static constexpr int A_TX = G * LINE * 16;
  static constexpr int B_BYTES = 9 * CIN * COUT * 2;
  static constexpr int ACC = (COUT + 31) / 32 * 32;          // TMEM columns per output line
  static constexpr int R = RR;                                // output lines per tile
  static constexpr int NSTG = 3 * (R + 2);                   // line stages per tile
  static constexpr uint32_t COLS = 2 * R * ACC <= 128 ? 128 : (2 * R * ACC <= 256 ? 256 : 512);
  static constexpr int NS_FIT = (200 * 1024 - 2 * B_BYTES - 128) / A_BYTES;
  static constexpr int NS = NS_FIT > R + 2 ? R + 2 : NS_FIT;
  static constexpr int SMEM = NS * A_BYTES + 2 * B_BYTES + 128;
  static constexpr uint32_t IDESC = idesc_bf16(TILE_M, COUT);
  static_assert(CIN % 16 == 0 && COUT % 16 == 0 && COUT <= 256, "channel counts");
  static_assert(NS >= 2 && NS <= R + 2, "ring depth (the weight-buffer reuse needs NS <= R + 2)");
  static_assert(2 * R * ACC <= 512, "TMEM columns");
  static_assert(B_BYTES % 128 == 0 && A_BYTES % 128 == 0, "stage alignment");
};

constexpr int PERSIST_THREADS = 192;

template <int CIN, int COUT, int RR>
__global__ void __launch_bounds__(PERSIST_THREADS, 1)
conv3_tc_persist_kernel(const __grid_constant__ CUtensorMap tmX,
                        const __nv_bfloat16* __restrict__ Wp, const float* __restrict__ bias,
                        void* __restrict__ Yv, const __nv_bfloat16* __restrict__ mask, int D,
                        int H, int W, int epi, int* err) {
  using C = PersistCfg<CIN, COUT, RR>;
  constexpr int NS = C::NS, R = C::R, NSTG = C::NSTG, ACC = C::ACC;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
  __shared__ __align__(8) uint64_t full[NS];
  __shared__ __align__(8) uint64_t empty[NS];
  __shared__ __align__(8) uint64_t acc_full[2];
  __shared__ __align__(8) uint64_t acc_empty[2];
  __shared__ __align__(8) uint64_t done;
  __shared__ uint32_t tmem_base;
  __shared__ volatile int failed;
  __shared__ int issued_s, consumed_s;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int n_wt = W / TILE_M, n_hb = (H + R - 1) / R;
  const int n_tiles = n_wt * n_hb * D;

  if (tid == 0) {
    for (int b = 0; b < NS; ++b) {
      mbar_init(&full[b], 1);
      mbar_init(&empty[b], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], 128);
    }
    mbar_init(&done, 1);
    failed = 0;
    issued_s = 0;
    consumed_s = 0;
    fence_barrier_init();
  }
  if (warp == 0) tmem_alloc(&tmem_base, C::COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base;
  uint8_t* const Bbase = smem + NS * C::A_BYTES;
  auto fail = [&](int code) {
    atomicOr(err, code);
    failed = 1;
  };

  if (warp == 0) {
    if (lane == 0) {  // producer
      int s = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < n_tiles && ok; t += gridDim.x) {
        const int w0 = (t % n_wt) * TILE_M, q = t / n_wt;
        const int h0 = (q % n_hb) * R, d = q / n_hb;
        for (int st = 0; st < NSTG; ++st, ++s) {
          const int buf = s % NS;
          if (s >= NS && !mbar_wait_f(&empty[buf], ((s / NS) - 1) & 1, &failed)) {
            fail(2);
            ok = false;
            break;
          }
          const int zi = st / (R + 2), ri = st % (R + 2);
          uint8_t* A = smem + buf * C::A_BYTES;
          const bool new_slice = ri == 0;
          mbar_expect_tx(&full[buf], C::A_TX + (new_slice ? C::B_BYTES : 0));
#pragma unroll
          for (int g = 0; g < C::G; ++g)
            tma_load_4d(A + g * CHUNK, &tmX, g * 8, w0 - 1, h0 - 1 + ri, d + zi - 1, &full[buf]);
          if (new_slice)
            bulk_load(Bbase + ((s / (R + 2)) & 1) * C::B_BYTES, Wp + (size_t)9 * zi * CIN * COUT,
                      C::B_BYTES, &full[buf]);
        }
      }
      issued_s = s;
    }
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      int s = 0, j = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < n_tiles && ok; t += gridDim.x, ++j) {
        const int b = j & 1;
        if (j >= 2 && !mbar_wait_f(&acc_empty[b], ((j >> 1) - 1) & 1, &failed)) {
          fail(8);
          break;
        }
        tc_fence_after();
        const uint32_t accb = tmem + (uint32_t)(b * R * ACC);
        for (int st = 0; st < NSTG; ++st, ++s) {
          const int buf = s % NS;
          if (!mbar_wait_f(&full[buf], (s / NS) & 1, &failed)) {
            fail(1);
            ok = false;
            break;
          }
          tc_fence_after();
          const int zi = st / (R + 2), ri = st % (R + 2);
          const uint64_t a_d = smem_desc(smem_u32(smem + buf * C::A_BYTES), CHUNK, 128);
          const uint64_t b_d =
              smem_desc(smem_u32(Bbase + ((s / (R + 2)) & 1) * C::B_BYTES), COUT * 16, 128);
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int dy = ri - 1 - r;  // input line h0-1+ri feeds output line h0+r
            if (dy < -1 || dy > 1) continue;
            const uint32_t td = accb + (uint32_t)(r * ACC);
#pragma unroll
            for (int dx = 0; dx < 3; ++dx) {
#pragma unroll
              for (int k = 0; k < CIN / 16; ++k) {
                const uint64_t ad = desc_add(a_d, 2 * k * CHUNK + dx * 16);
                const uint64_t bd =
                    desc_add(b_d, ((3 * (dy + 1) + dx) * C::G + 2 * k) * COUT * 16);
                // the first product into line r (zi 0, dy -1, dx 0, k 0) overwrites
                const uint32_t acc = (zi != 0 || dy != -1 || dx != 0 || k != 0) ? 1u : 0u;
                mma_bf16(td, ad, bd, C::IDESC, acc);
              }
            }
          }
          mma_commit(&empty[buf]);
        }
        if (!ok) break;
        mma_commit(&acc_full[b]);
      }
      consumed_s = s;
      // every product issued has completed before the CTA releases TMEM
      mma_commit(&done);
      if (!mbar_wait(&done, 0)) atomicOr(err, 4);
    }
  } else {  // epilogue: warps 2-5, TMEM lane quarter warp & 3
    const int row = (warp & 3) * 32 + lane;
    const uint32_t tlane = tmem + ((uint32_t)((warp & 3) * 32) << 16);
    int j = 0;
    for (int t = blockIdx.x; t < n_tiles; t += gridDim.x, ++j) {
      const int b = j & 1;
      if (!mbar_wait_sleep(&acc_full[b], (j >> 1) & 1, &failed)) {
        if (lane == 0) fail(16);
        break;
      }
      tc_fence_after();
      const int w0 = (t % n_wt) * TILE_M, q = t / n_wt;
      const int h0 = (q % n_hb) * R, d = q / n_hb;
#pragma unroll 1
      for (int r = 0; r < R; ++r) {
        if (h0 + r >= H) break;
        const uint32_t tl = tlane + (uint32_t)(b * R * ACC + r * ACC);
        const int64_t vox = ((int64_t)d * H + h0 + r) * W + w0 + row;
        if (epi == EPI_F32_C0) {
          float v[16];
          tmem_ld16(tl, v);
          ((float*)Yv)[vox] = v[0] + bias[0];
        } else {
          __nv_bfloat16* Y = (__nv_bfloat16*)Yv;
#pragma unroll
          for (int c0 = 0; c0 < COUT; c0 += 16) {
            float v[16];
            tmem_ld16(tl + c0, v);
            __align__(16) __nv_bfloat16 o[16];
            if (epi == EPI_MASK) {
              const uint4* mp = (const uint4*)(mask + vox * COUT + c0);
              __align__(16) __nv_bfloat16 m[16];
              *(uint4*)&m[0] = mp[0];
              *(uint4*)&m[8] = mp[1];
#pragma unroll
              for (int qq = 0; qq < 16; ++qq)
                o[qq] = __float2bfloat16(__bfloat162float(m[qq]) > 0.0f ? v[qq] : 0.0f);
            } else {
#pragma unroll
              for (int qq = 0; qq < 16; ++qq) {
                float y = v[qq] + bias[c0 + qq];
                if (epi == EPI_RELU) y = fmaxf(y, 0.0f);
                o[qq] = __float2bfloat16(y);
              }
            }
            uint4* yp = (uint4*)(Y + vox * COUT + c0);
            yp[0] = *(uint4*)&o[0];
            yp[1] = *(uint4*)&o[8];
          }
        }
      }
      tc_fence_before();
      mbar_arrive(&acc_empty[b]);
    }
  }
  __syncthreads();
  if (tid == 0 && failed) {
    // let the copies already issued land before the CTA releases its smem
    for (int s = consumed_s; s < issued_s; ++s) (void)mbar_wait(&full[s % NS], (s / NS) & 1);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, C::COLS);
}

// -------------------------------------------------------------------------
// host side: tensor maps and dispatch

static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

static hp_status get_encode() {
  static std::once_flag once;
  static cudaError_t st = cudaSuccess;
  std::call_once(once, [] {
    cudaDriverEntryPointQueryResult q;
    void* fn = nullptr;
    st = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    if (st == cudaSuccess && q == cudaDriverEntryPointSuccess) g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  });
  if (!g_encode) {
    hp::set_error("cuTensorMapEncodeTiled is not available");
    return HP_ERR_CUDA;
  }
  return HP_OK;
}

// Tensor map over X[D][H][W][C] (bf16) with box (8 ch, box_w voxels, 1, 1).
hp_status make_line_map(CUtensorMap* map, const void* X, int D, int H, int W, int Cch,
                        int box_w = LINE) {
  hp_status s = get_encode();
  if (s != HP_OK) return s;
  if (((uintptr_t)X & 15) != 0) {
    hp::set_error("conv input must be 16-byte aligned");
    return HP_ERR_INVALID;
  }
  cuuint64_t dims[4] = {(cuuint64_t)Cch, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)D};
  cuuint64_t strides[3] = {(cuuint64_t)Cch * 2, (cuuint64_t)W * Cch * 2,
                           (cuuint64_t)H * W * Cch * 2};
  cuuint32_t box[4] = {8, (cuuint32_t)box_w, 1, 1};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  CUresult r = g_encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, (void*)X, dims, strides, box,
                        estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    hp::set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
    return HP_ERR_CUDA;
  }
  return HP_OK;
}

typedef void (*ConvFn)(CUtensorMap, const __nv_bfloat16*, const float*, void*,
                       const __nv_bfloat16*, int, int, int, int, int*);

struct ConvEntry {
  int cin, cout, smem;
  ConvFn fn;
  int rows_smem;
  ConvFn rows_fn;   // CONV_ROWS output lines per CTA
  int persist_smem;
  ConvFn persist_fn;   // persistent warp-specialised kernel, or null
  int persist_rows;
  uint32_t persist_cols;
};

// Kernel per layer shape, from per-shape timings on B200 (network level
// sizes, hp_conv3_forward, CUDA events): the persistent kernel with two
// output lines per tile wins on the wide layers (96 -> 32 95 against
// 134 us, 32 -> 96 55 against 73, 64 -> 64 29 against 35, 64 -> 32 25
// against 31) and loses on the narrow ones (16 -> 16 108-118 against 54,
// 48 -> 16 195 against 125, 32 -> 32 49 against 35): one CTA per SM
// pair of copy and MMA threads keeps fewer small products in flight than
// four row-blocked CTAs.
#define HP_CONV(ci, co)                                                                     \
  {ci, co, ConvCfg<ci, co>::SMEM, conv3_tc_kernel<ci, co>, RowsCfg<ci, co, CONV_ROWS>::SMEM, \
   conv3_tc_rows_kernel<ci, co, CONV_ROWS>, 0, nullptr, 0, 0}
#define HP_CONV_P(ci, co)                                                                   \
  {ci, co, ConvCfg<ci, co>::SMEM, conv3_tc_kernel<ci, co>, RowsCfg<ci, co, CONV_ROWS>::SMEM, \
   conv3_tc_rows_kernel<ci, co, CONV_ROWS>, PersistCfg<ci, co, 2>::SMEM,                    \
   conv3_tc_persist_kernel<ci, co, 2>, 2, PersistCfg<ci, co, 2>::COLS}
static const ConvEntry kConv[] = {
    HP_CONV(16, 16),   HP_CONV(16, 32),   HP_CONV(32, 16),   HP_CONV(32, 32), HP_CONV(32, 64),
    HP_CONV_P(64, 32), HP_CONV_P(64, 64), HP_CONV(48, 16),   HP_CONV_P(96, 32), HP_CONV(16, 48),
    HP_CONV_P(32, 96),
};
#undef HP_CONV
#undef HP_CONV_P

hp_status conv3_launch(const void* X, const void* Wp, const float* bias, void* Y,
                       const void* mask, int D, int H, int W, int cin, int cout, int epi,
                       int* err, cudaStream_t s) {
  const ConvEntry* e = nullptr;
  for (const auto& c : kConv)
    if (c.cin == cin && c.cout == cout) e = &c;
  if (!e) {
    hp::set_error("conv %d->%d is not compiled", cin, cout);
    return HP_ERR_UNSUPPORTED;
  }
  if (W % TILE_M != 0 || D < 1 || H < 1) {
    hp::set_error("conv grid W=%d must be a multiple of %d", W, TILE_M);
    return HP_ERR_INVALID;
  }
  if (((uintptr_t)Wp & 15) || ((uintptr_t)Y & 15) || (mask && ((uintptr_t)mask & 15))) {
    hp::set_error("conv buffers must be 16-byte aligned");
    return HP_ERR_INVALID;
  }
  CUtensorMap map;
  hp_status st = make_line_map(&map, X, D, H, W, cin);
  if (st != HP_OK) return st;
  static bool attr_set[sizeof(kConv) / sizeof(kConv[0])] = {false};
  static int persist_grid[sizeof(kConv) / sizeof(kConv[0])] = {0};
  const int idx = (int)(e - kConv);
  if (!attr_set[idx]) {
    HP_CUDA_TRY(cudaFuncSetAttribute((const void*)e->fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     e->smem));
    HP_CUDA_TRY(cudaFuncSetAttribute((const void*)e->rows_fn,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, e->rows_smem));
    if (e->persist_fn) {
      HP_CUDA_TRY(cudaFuncSetAttribute((const void*)e->persist_fn,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       e->persist_smem));
      // resident CTAs of the persistent kernel: shared memory and TMEM columns
      int dev = 0, n_sm = 0, per_sm = 0;
      HP_CUDA_TRY(cudaGetDevice(&dev));
      HP_CUDA_TRY(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
      HP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &per_sm, (const void*)e->persist_fn, PERSIST_THREADS, e->persist_smem));
      per_sm = std::min(per_sm, (int)(512 / e->persist_cols));
      persist_grid[idx] = std::max(1, per_sm) * n_sm;
    }
    attr_set[idx] = true;
  }
  if (e->persist_fn) {
    const int n_tiles = (W / TILE_M) * ((H + e->persist_rows - 1) / e->persist_rows) * D;
    const int grid = std::min(n_tiles, persist_grid[idx]);
    e->persist_fn<<<grid, PERSIST_THREADS, e->persist_smem, s>>>(
        map, (const __nv_bfloat16*)Wp, bias, Y, (const __nv_bfloat16*)mask, D, H, W, epi, err);
    HP_CUDA_TRY(cudaGetLastError());
    return HP_OK;
  }
  // Row-blocked CTAs where their two line stages and two weight slices stay
  // small enough for several CTAs per SM; the wide layers (64+ input or
  // output channels with large weight slices) keep one line per CTA, which
  // measured faster there on B200 (e.g. 96 -> 32: 135 vs 156 us).
  if (e->rows_smem <= 64 * 1024) {
    dim3 grid(W / TILE_M, (H + CONV_ROWS - 1) / CONV_ROWS, D);
    e->rows_fn<<<grid, 128, e->rows_smem, s>>>(map, (const __nv_bfloat16*)Wp, bias, Y,
                                               (const __nv_bfloat16*)mask, D, H, W, epi, err);
  } else {
    dim3 grid(W / TILE_M, H, D);
    e->fn<<<grid, 128, e->smem, s>>>(map, (const __nv_bfloat16*)Wp, bias, Y,
                                     (const __nv_bfloat16*)mask, D, H, W, epi, err);
  }
  HP_CUDA_TRY(cudaGetLastError());
  return HP_OK;
}


// -------------------------------------------------------------------------
// Weight gradient of a 3x3x3 layer on the tensor cores:
//   gw[co][ci][t] = sum_v G[v][co] X[v + off(t)][ci],  gb[co] = sum_v G[v][co]
// as GEMMs with K = voxels.  The [voxel][8-channel] line tiles that TMA
// brings in for the forward pass are, read transposed, MN-major UMMA
// operands: a core matrix is 8 voxel rows (K) of 16 bytes (8 channels), K
// groups 128 bytes apart, channel groups one tile chunk apart.  A CTA owns
// one dz and a range of output lines (d, h, 128 voxels along W); per line
// it loads the three input lines (d+dz, h-1..h+1) of X (130 voxels with the
// halo, zero-filled outside the grid) as 3 CIN/8 chunk slots and the G line
// as N/8 chunks.  The slots form M tiles of 128 rows (16 slots; rows past
// the last slot read zeroed slots), and the three dx taps are the same tile
// with the descriptor start moved by one voxel row (16 bytes), as in the
// forward kernel.  Each (M tile, dx) accumulates over the CTA's lines in
// its own TMEM columns (M = 128 rows, N = padded COUT, FP32).  The CTAs'
// partial sums go to a workspace and a second kernel adds them in a fixed
// order: the result does not depend on scheduling (no atomics).
template <int CIN, int N>
struct WgCfg {
  static constexpr int G = CIN / 8;              // chunks per input line
  static constexpr int S = 3 * G;                // loaded slots per line (dy = -1, 0, 1)
  static constexpr int T = (S + 15) / 16;        // M tiles of 128 rows
  static constexpr int A_BYTES = 16 * T * CHUNK;
  static constexpr int A_TX = S * LINE * 16;
  static constexpr int B_BYTES = (N / 8) * TILE_M * 16;
  static constexpr int STAGE = A_BYTES + B_BYTES;
  static constexpr int SMEM = 2 * STAGE + 128;
  static constexpr int ACC = 3 * T * N;          // TMEM columns of the accumulators
  static constexpr uint32_t COLS =
      ACC <= 32 ? 32 : (ACC <= 64 ? 64 : (ACC <= 128 ? 128 : (ACC <= 256 ? 256 : 512)));
  // BF16 x BF16 -> FP32, M = 128, both operands MN-major (bits 15 and 16)
  static constexpr uint32_t IDESC = idesc_bf16(TILE_M, N) | (1u << 15) | (1u << 16);
  static_assert(CIN % 8 == 0 && N % 16 == 0 && N <= 256, "channel counts");
  static_assert(ACC <= 512, "TMEM columns");
  static_assert(SMEM <= 227 * 1024, "shared memory");
  static_assert(A_BYTES % 128 == 0 && B_BYTES % 128 == 0, "stage alignment");
};

template <int CIN, int N>
__global__ void __launch_bounds__(128)
wgrad3_tc_kernel(const __grid_constant__ CUtensorMap tmX, const __grid_constant__ CUtensorMap tmG,
                 int D, int H, int WT, int lines_per_cta, float* __restrict__ part, int* err) {
  using C = WgCfg<CIN, N>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
  __shared__ __align__(8) uint64_t full[2];
  __shared__ __align__(8) uint64_t empty[2];
  __shared__ __align__(8) uint64_t done;
  __shared__ uint32_t tmem_base;
  __shared__ int failed;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int dz = (int)blockIdx.y - 1;
  const int nl = D * H * WT;
  const int l0 = blockIdx.x * lines_per_cta;
  const int l1 = min(nl, l0 + lines_per_cta);

  // the slots past the loaded ones are read by the last M tile: zero them
  // in both stages (the TMA never writes them)
  for (int buf = 0; buf < 2; ++buf) {
    uint4* z = (uint4*)(smem + buf * C::STAGE + C::S * CHUNK);
    const int n16 = (16 * C::T - C::S) * CHUNK / 16;
    for (int q = tid; q < n16; q += 128) z[q] = make_uint4(0u, 0u, 0u, 0u);
  }
  fence_proxy_async();
  if (tid == 0) {
    mbar_init(&full[0], 1);
    mbar_init(&full[1], 1);
    mbar_init(&empty[0], 1);
    mbar_init(&empty[1], 1);
    mbar_init(&done, 1);
    failed = 0;
    fence_barrier_init();
  }
  if (warp == 0) tmem_alloc(&tmem_base, C::COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base;
  const int nmine = max(0, l1 - l0);

  if (tid == 0 && nmine > 0) {
    auto issue = [&](int li, int buf) {
      const int wt = li % WT, h = (li / WT) % H, d = li / (WT * H);
      uint8_t* A = smem + buf * C::STAGE;
      uint8_t* B = A + C::A_BYTES;
      mbar_expect_tx(&full[buf], C::A_TX + C::B_BYTES);
#pragma unroll
      for (int dy = 0; dy < 3; ++dy)
#pragma unroll
        for (int g = 0; g < C::G; ++g)
          tma_load_4d(A + (dy * C::G + g) * CHUNK, &tmX, g * 8, wt * TILE_M - 1, h + dy - 1,
                      d + dz, &full[buf]);
#pragma unroll
      for (int g = 0; g < N / 8; ++g)
        tma_load_4d(B + g * TILE_M * 16, &tmG, g * 8, wt * TILE_M, h, d, &full[buf]);
    };
    int issued = 0, consumed = 0;
    issue(l0, 0);
    issued = 1;
    if (nmine > 1) {
      issue(l0 + 1, 1);
      issued = 2;
    }
    for (int s = 0; s < nmine; ++s) {
      const int buf = s & 1;
      const uint32_t par = (s >> 1) & 1;
      if (!mbar_wait(&full[buf], par)) {
        atomicOr(err, 8);
        failed = 1;
        break;
      }
      tc_fence_after();
      const uint32_t a0 = smem_u32(smem + buf * C::STAGE);
      const uint32_t b0 = a0 + C::A_BYTES;
#pragma unroll
      for (int t = 0; t < C::T; ++t) {
#pragma unroll
        for (int dx = 0; dx < 3; ++dx) {
#pragma unroll
          for (int k = 0; k < TILE_M / 16; ++k) {
            const uint64_t ad = smem_desc(a0 + 16 * t * CHUNK + dx * 16 + k * 256, 128, CHUNK);
            const uint64_t bd = smem_desc(b0 + k * 256, 128, TILE_M * 16);
            mma_bf16(tmem + (uint32_t)((t * 3 + dx) * N), ad, bd, C::IDESC, (s | k) != 0);
          }
        }
      }
      mma_commit(&empty[buf]);
      consumed = s + 1;
      if (s + 2 < nmine) {
        if (!mbar_wait(&empty[buf], par)) {
          atomicOr(err, 16);
          failed = 1;
          break;
        }
        issue(l0 + s + 2, buf);
        ++issued;
      }
    }
    if (failed) {
      for (int s = consumed; s < issued; ++s) (void)mbar_wait(&full[s & 1], (s >> 1) & 1);
    }
  }
  if (tid == 0) mma_commit(&done);
  __syncthreads();
  const bool ok = mbar_wait(&done, 0) && !failed;
  if (!ok && tid == 0) atomicOr(err, 32);
  tc_fence_after();
  // epilogue: TMEM lane tid = GEMM row tid of every (M tile, dx)
  const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
  const int64_t base = ((int64_t)blockIdx.y * gridDim.x + blockIdx.x) * (C::T * 3);
#pragma unroll 1
  for (int q = 0; q < C::T * 3; ++q) {
    float* dst = part + ((base + q) * TILE_M + tid) * N;
#pragma unroll
    for (int c0 = 0; c0 < N; c0 += 16) {
      float v[16];
      if (ok && nmine > 0) {
        tmem_ld16(trow + (uint32_t)(q * N + c0), v);
      } else {
#pragma unroll
        for (int u = 0; u < 16; ++u) v[u] = 0.0f;
      }
#pragma unroll
      for (int u = 0; u < 16; u += 4) *(float4*)(dst + c0 + u) = make_float4(v[u], v[u + 1], v[u + 2], v[u + 3]);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, C::COLS);
}

// Per-block partial sums of G over voxels (bias gradient), fixed order:
// thread (r, co) sums voxels r, r + R, ... of the block's range, then the
// block adds its R rows in order.
constexpr int GS_BLOCKS = 256;
__global__ void __launch_bounds__(256)
gsum_partial_kernel(const __nv_bfloat16* __restrict__ G, int64_t n, int coP, float* __restrict__ part) {
  __shared__ float sh[256];
  const int R = 256 / coP;
  const int r = threadIdx.x / coP, co = threadIdx.x % coP;
  const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
  const int64_t v0 = blockIdx.x * chunk, v1 = min(n, v0 + chunk);
  float acc = 0.0f;
  if (r < R)
    for (int64_t v = v0 + r; v < v1; v += R) acc += __bfloat162float(G[v * coP + co]);
  sh[threadIdx.x] = r < R ? acc : 0.0f;
  __syncthreads();
  if (threadIdx.x < coP) {
    float s = 0.0f;
    for (int q = 0; q < R; ++q) s += sh[q * coP + threadIdx.x];
    part[(int64_t)blockIdx.x * coP + threadIdx.x] = s;
  }
}

// gw[co][ci][t] and gb[co] from the partials, each summed in CTA order.
template <int CIN, int N>
__global__ void __launch_bounds__(256)
wgrad_reduce_kernel(const float* __restrict__ part, int nchunk, const float* __restrict__ gpart,
                    int cout, float* __restrict__ gw, float* __restrict__ gb) {
  using C = WgCfg<CIN, N>;
  const int64_t nw = (int64_t)cout * CIN * 27;
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e < nw) {
    const int t = (int)(e % 27), ci = (int)((e / 27) % CIN), co = (int)(e / (27 * CIN));
    const int dzi = t / 9, dy = (t / 3) % 3, dx = t % 3;
    const int slot = dy * C::G + ci / 8;
    const int mt = slot / 16, row = (slot % 16) * 8 + ci % 8;
    float s = 0.0f;
    for (int c = 0; c < nchunk; ++c) {
      const int64_t q = ((int64_t)dzi * nchunk + c) * (C::T * 3) + mt * 3 + dx;
      s += part[(q * TILE_M + row) * N + co];
    }
    gw[e] = s;
  } else if (e < nw + cout) {
    const int co = (int)(e - nw);
    float s = 0.0f;
    for (int b = 0; b < GS_BLOCKS; ++b) s += gpart[(int64_t)b * N + co];
    gb[co] = s;
  }
}

static int wg_chunks(int nl) {
  // about two CTAs per SM over the three dz slices, at least one line each
  const int target = 100;
  const int per = std::max(1, (nl + target - 1) / target);
  return (nl + per - 1) / per;
}

int64_t wgrad3_workspace(int D, int H, int W, int cin, int cout) {
  const int N = cout < 16 ? 16 : cout;
  const int T = (3 * (cin / 8) + 15) / 16;
  const int nl = D * H * std::max(1, W / TILE_M);
  return (int64_t)3 * wg_chunks(nl) * T * 3 * TILE_M * N * 4 + (int64_t)GS_BLOCKS * N * 4;
}

typedef void (*WgFn)(CUtensorMap, CUtensorMap, int, int, int, int, float*, int*);
typedef void (*WgRedFn)(const float*, int, const float*, int, float*, float*);
struct WgEntry {
  int cin, n, smem;
  WgFn fn;
  WgRedFn red;
};
#define HP_WG(ci, n) {ci, n, WgCfg<ci, n>::SMEM, wgrad3_tc_kernel<ci, n>, wgrad_reduce_kernel<ci, n>}
static const WgEntry kWg[] = {
    HP_WG(16, 16), HP_WG(16, 32), HP_WG(32, 32), HP_WG(32, 64), HP_WG(64, 64), HP_WG(96, 32),
    HP_WG(48, 16), HP_WG(32, 16), HP_WG(64, 32),
};
#undef HP_WG

hp_status wgrad3_launch(const void* X, const void* G, int D, int H, int W, int cin, int cout,
                        float* gw, float* gb, void* work, int64_t work_bytes, int* err,
                        cudaStream_t s) {
  const int N = cout < 16 ? 16 : cout;
  const WgEntry* e = nullptr;
  for (const auto& c : kWg)
    if (c.cin == cin && c.n == N) e = &c;
  if (!e) {
    hp::set_error("weight gradient %d->%d is not compiled", cin, cout);
    return HP_ERR_UNSUPPORTED;
  }
  if (W % TILE_M != 0 || D < 1 || H < 1) {
    hp::set_error("weight gradient grid W=%d must be a multiple of %d", W, TILE_M);
    return HP_ERR_INVALID;
  }
  if (((uintptr_t)G & 15) || ((uintptr_t)work & 15)) {
    hp::set_error("weight gradient buffers must be 16-byte aligned");
    return HP_ERR_INVALID;
  }
  const int64_t need = wgrad3_workspace(D, H, W, cin, cout);
  if (work_bytes < need) {
    hp::set_error("weight gradient workspace of %lld bytes is below the %lld needed",
                  (long long)work_bytes, (long long)need);
    return HP_ERR_INVALID;
  }
  CUtensorMap mx, mg;
  hp_status st = make_line_map(&mx, X, D, H, W, cin, LINE);
  if (st != HP_OK) return st;
  st = make_line_map(&mg, G, D, H, W, N, TILE_M);
  if (st != HP_OK) return st;
  static bool attr_set[sizeof(kWg) / sizeof(kWg[0])] = {false};
  const int idx = (int)(e - kWg);
  if (!attr_set[idx]) {
    HP_CUDA_TRY(cudaFuncSetAttribute((const void*)e->fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     e->smem));
    attr_set[idx] = true;
  }
  const int WT = W / TILE_M;
  const int nl = D * H * WT;
  const int nchunk = wg_chunks(nl);
  const int per = (nl + nchunk - 1) / nchunk;
  float* part = (float*)work;
  const int T = (3 * (cin / 8) + 15) / 16;
  float* gpart = part + (int64_t)3 * nchunk * T * 3 * TILE_M * N;
  e->fn<<<dim3(nchunk, 3), 128, e->smem, s>>>(mx, mg, D, H, WT, per, part, err);
  HP_CUDA_TRY(cudaGetLastError());
  gsum_partial_kernel<<<GS_BLOCKS, 256, 0, s>>>((const __nv_bfloat16*)G, (int64_t)D * H * W, N,
                                                gpart);
  HP_CUDA_TRY(cudaGetLastError());
  const int64_t nout = (int64_t)cout * cin * 27 + cout;
  e->red<<<(unsigned)((nout + 255) / 256), 256, 0, s>>>(part, nchunk, gpart, cout, gw, gb);
  HP_CUDA_TRY(cudaGetLastError());
  return HP_OK;
}

}  // namespace tc
}  // namespace hp

// Test / building-block entry point: one 3x3x3 convolution (zero padding 1).
extern "C" hp_status hp_conv3_forward(const void* X, const void* Wp, const float* bias, void* Y,
                                      const void* mask, int32_t D, int32_t H, int32_t W,
                                      int32_t cin, int32_t cout, int32_t epi, int32_t* err,
                                      void* stream) {
  HP_REQUIRE(X && Wp && Y && err && (bias || epi == hp::tc::EPI_MASK),
             "hp_conv3_forward: null argument");
  HP_REQUIRE(epi >= 0 && epi <= 3, "hp_conv3_forward: bad epilogue %d", epi);
  HP_REQUIRE(epi != hp::tc::EPI_MASK || mask, "hp_conv3_forward: mask epilogue needs mask");
  return hp::tc::conv3_launch(X, Wp, bias, Y, mask, D, H, W, cin, cout, epi, err,
                              (cudaStream_t)stream);
}

extern "C" int64_t hp_conv3_wgrad_workspace(int32_t D, int32_t H, int32_t W, int32_t cin,
                                            int32_t cout) {
  if (D < 1 || H < 1 || W < 1 || cin < 8 || cout < 1) return -1;
  return hp::tc::wgrad3_workspace(D, H, W, cin, cout);
}

extern "C" hp_status hp_conv3_wgrad(const void* X, const void* G, int32_t D, int32_t H, int32_t W,
                                    int32_t cin, int32_t cout, float* gw, float* gb, void* work,
                                    int64_t work_bytes, int32_t* err, void* stream) {
  HP_REQUIRE(X && G && gw && gb && work && err, "hp_conv3_wgrad: null argument");
  return hp::tc::wgrad3_launch(X, G, D, H, W, cin, cout, gw, gb, work, work_bytes, err,
                               (cudaStream_t)stream);
}
