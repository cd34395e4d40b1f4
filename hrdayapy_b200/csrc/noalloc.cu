// Allocation-free FP64 true-residual check of a torso potential field.
//
// Some callers cannot allocate device memory while they work: code running
// inside a host framework that owns every device allocation through its own
// pool, real-time loops that must not enter the driver's allocator, or
// callers bound by a fixed memory budget.  hp_torso_residual_noalloc gives
// them the solver's convergence judge -- ||b - A x|| and ||b|| in FP64 over
// the torso operator -- without any cudaMalloc: the only scratch it needs
// (the per-block partial sums of a deterministic reduction, a ticket
// counter and two error counters) lives in the file-scope array
// g_noalloc_scratch below.
//
// Limits and sharing:
//   * at most HP_NOALLOC_MAX_CELLS padded grid cells per call (one thread
//     per cell, one partial per 256-cell block);
//   * the array exists once per GPU that loads the library and stays
//     allocated until the process exits: (4 + 2 * HP_NOALLOC_MAX_BLOCKS)
//     doubles = 1,048,608 bytes (about 1.0 MiB);
//   * every call on a device uses the same array, which keeps the last
//     call's contents: the ticket and the error counters are cleared at the
//     start of each call, so sequential calls are independent, but calls
//     that overlap on the GPU (concurrent streams, or host threads calling
//     at once) race and must not be issued;
//   * the call is synchronous: it copies its two sums back to the host and
//     waits for the stream before it returns;
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current and keeps it for the
//     life of the process, so make that first call before any stream
//     capture begins, and do not use the entry point across a
//     cudaDeviceReset (the kept address belongs to the old context).
#include "hp_common.cuh"

#include <math.h>
#include <mutex>

namespace hp {
namespace noalloc {

constexpr int TB = 256;
constexpr int64_t MAX_CELLS = (int64_t)HP_NOALLOC_MAX_BLOCKS * TB;
constexpr int MAX_DEVICES = 64;

// [0] ticket (uint32) + count of interior voxels with a label >= n_materials
// (uint32), [1] ||r||^2, [2] ||b||^2, [3] count of border cells that are not
// air (uint32), [4 + 2 q], [5 + 2 q]: partials of block q.
static __device__ __align__(256) double g_noalloc_scratch[4 + 2 * HP_NOALLOC_MAX_BLOCKS];

struct Params {
  int32_t pi, pj, pk;          // padded dims
  int64_t ng;
  int64_t pin;
  int32_t n_materials;
  double sigma[HP_MAX_MATERIALS];
  double inv_h2;
};

__device__ __forceinline__ double face(const Params& p, int u, int v) {
  if (u == 0 || v == 0) return 0.0;
  const double su = p.sigma[u], sv = p.sigma[v];
  if (su + sv < 1e-30) return 0.0;
  return (2.0 * su * sv) / (su + sv) * p.inv_h2;
}

__global__ void __launch_bounds__(TB)
residual_kernel(Params p, const uint8_t* __restrict__ label, const double* __restrict__ x,
                const float* __restrict__ b, double* scratch) {
  unsigned int* ticket = (unsigned int*)scratch;
  unsigned int* bad = ticket + 1;
  unsigned int* bad_border = (unsigned int*)(scratch + 3);
  const int64_t g = blockIdx.x * (int64_t)TB + threadIdx.x;
  double rr = 0.0, bb = 0.0;
  if (g < p.ng) {
    const int64_t SJ = p.pk, SI = (int64_t)p.pj * p.pk;
    const int i = (int)(g / SI), j = (int)((g / SJ) % p.pj), k = (int)(g % SJ);
    const bool interior = i > 0 && i < p.pi - 1 && j > 0 && j < p.pj - 1 && k > 0 && k < p.pk - 1;
    const int l = label[g];
    if (!interior && l != 0) atomicAdd(bad_border, 1u);
    if (interior && l != 0 && g != p.pin) {
      if (l >= p.n_materials) {
        atomicAdd(bad, 1u);
      } else {
        const int64_t nb[6] = {g + SI, g - SI, g + SJ, g - SJ, g + 1, g - 1};
        const double xg = x[g];
        double ax = 0.0;   // face-flux form, as the solver's true residual
#pragma unroll
        for (int f = 0; f < 6; ++f) {
          const int ln = label[nb[f]];
          const double t = ln < p.n_materials ? face(p, l, ln) : 0.0;
          ax += t * (xg - x[nb[f]]);
        }
        const double bv = (double)b[g];
        const double r = bv - ax;
        rr = r * r;
        bb = bv * bv;
      }
    }
  }
  // block reduction (fixed order), then the last block sums the partials
  __shared__ double s_rr[TB], s_bb[TB];
  __shared__ bool last;
  s_rr[threadIdx.x] = rr;
  s_bb[threadIdx.x] = bb;
  __syncthreads();
  for (int s = TB / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      s_rr[threadIdx.x] += s_rr[threadIdx.x + s];
      s_bb[threadIdx.x] += s_bb[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    scratch[4 + 2 * (int64_t)blockIdx.x] = s_rr[0];
    scratch[5 + 2 * (int64_t)blockIdx.x] = s_bb[0];
    __threadfence();
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double a = 0.0, c = 0.0;
  for (int q = threadIdx.x; q < (int)gridDim.x; q += TB) {
    a += ((volatile double*)scratch)[4 + 2 * q];
    c += ((volatile double*)scratch)[5 + 2 * q];
  }
  s_rr[threadIdx.x] = a;
  s_bb[threadIdx.x] = c;
  __syncthreads();
  for (int s = TB / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      s_rr[threadIdx.x] += s_rr[threadIdx.x + s];
      s_bb[threadIdx.x] += s_bb[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    scratch[1] = s_rr[0];
    scratch[2] = s_bb[0];
    *ticket = 0u;
  }
}

// Device address of g_noalloc_scratch, looked up once per device.
static double* g_ptr[MAX_DEVICES] = {nullptr};
static std::mutex g_mu;

static hp_status scratch_ptr(double** out) {
  int dev = 0;
  HP_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= MAX_DEVICES) {
    hp::set_error("hp_torso_residual_noalloc: device %d beyond the supported %d", dev,
                  MAX_DEVICES);
    return HP_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      hp::set_error("hp_torso_residual_noalloc: cudaGetSymbolAddress failed: %s",
                    cudaGetErrorString(e));
      return HP_ERR_CUDA;
    }
    g_ptr[dev] = (double*)p;
  }
  *out = g_ptr[dev];
  return HP_OK;
}

}  // namespace noalloc
}  // namespace hp

extern "C" hp_status hp_torso_residual_noalloc(int32_t ni, int32_t nj, int32_t nk,
                                               const uint8_t* label, const double* sigma,
                                               int32_t n_materials, double h_m,
                                               int64_t pin_cell, const double* x,
                                               const float* b, double* out, void* stream) {
  using namespace hp::noalloc;
  HP_REQUIRE(label && sigma && x && b && out, "hp_torso_residual_noalloc: null argument");
  HP_REQUIRE(ni > 0 && nj > 0 && nk > 0, "hp_torso_residual_noalloc: empty grid");
  HP_REQUIRE(n_materials >= 1 && n_materials <= HP_MAX_MATERIALS,
             "hp_torso_residual_noalloc: n_materials must be 1..%d", HP_MAX_MATERIALS);
  HP_REQUIRE(h_m > 0.0, "hp_torso_residual_noalloc: h_m must be positive");
  const int64_t ng = ((int64_t)ni + 2) * ((int64_t)nj + 2) * ((int64_t)nk + 2);
  HP_REQUIRE(ng <= MAX_CELLS,
             "hp_torso_residual_noalloc: padded grid of %lld cells exceeds the maximum of %lld "
             "cells (its scratch array is fixed at build time)",
             (long long)ng, (long long)MAX_CELLS);
  HP_REQUIRE(pin_cell >= -1 && pin_cell < ng, "hp_torso_residual_noalloc: pin_cell out of range");
  double* scratch = nullptr;
  hp_status st = scratch_ptr(&scratch);
  if (st != HP_OK) return st;
  Params p;
  p.pi = ni + 2;
  p.pj = nj + 2;
  p.pk = nk + 2;
  p.ng = ng;
  p.pin = pin_cell;
  p.n_materials = n_materials;
  for (int q = 0; q < HP_MAX_MATERIALS; ++q) p.sigma[q] = q < n_materials ? sigma[q] : 0.0;
  p.inv_h2 = 1.0 / (h_m * h_m);
  cudaStream_t s = (cudaStream_t)stream;
  // the ticket and both error counters must start at zero (words 0-3)
  HP_CUDA_TRY(cudaMemsetAsync(scratch, 0, 4 * sizeof(double), s));
  const unsigned int nblk = (unsigned int)((ng + TB - 1) / TB);
  residual_kernel<<<nblk, TB, 0, s>>>(p, label, x, b, scratch);
  HP_CUDA_TRY(cudaGetLastError());
  double res[4];
  HP_CUDA_TRY(cudaMemcpyAsync(res, scratch, 4 * sizeof(double), cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  unsigned int bad = ((unsigned int*)&res[0])[1];
  unsigned int bad_border = ((unsigned int*)&res[3])[0];
  if (bad_border) {
    hp::set_error("hp_torso_residual_noalloc: %u cells of the one-voxel border carry a nonzero "
                  "label; the border of the padded grid must be air (label 0)", bad_border);
    return HP_ERR_INVALID;
  }
  if (bad) {
    hp::set_error("hp_torso_residual_noalloc: %u voxels carry a label >= n_materials", bad);
    return HP_ERR_INVALID;
  }
  out[0] = sqrt(res[1]);
  out[1] = sqrt(res[2]);
  return HP_OK;
}
