// Learned preconditioner for the torso Poisson solve (no counterpart in the
// reference, whose solver is Jacobi-PCG only).
//
//   M(r) = omega * D^-1 r  +  Q A_c^-1 Q^T r  +  P( s * CNN( [R(D^-1 r) / s, geometry] ) )
//
// Q is piecewise-constant aggregation over cubes of ag^3 torso voxels and
// A_c = Q^T A Q the Galerkin coarse operator (a few thousand unknowns at
// most), factorised and inverted once on the host and applied as a dense
// mat-vec: it removes the global, smooth error modes that Jacobi leaves and
// that no network with a local receptive field can represent.  The network
// learns what remains between the two scales.  Without the network
// (use_net = 0) M is the same two-level preconditioner, so the network's
// gain is measured against exactly the method without it.
//
// R restricts the fine torso grid (padded, see torso.cu) by 2 x 2 x 2
// averaging onto the network grid (half resolution, NDHWC BF16, 16 input
// channels: the Jacobi-scaled residual normalised by its RMS s, the active
// fraction and the per-material fractions of each coarse cell); P is the
// piecewise-constant prolongation back to the active fine cells.  The CNN is
// a 3-level encoder-decoder with 16 / 32 / 64 channels, 3x3x3 convolutions
// (tcgen05 implicit GEMM, BF16 operands, FP32 accumulation, csrc/conv.cu),
// ReLU, 2 x 2 average pooling / nearest upsampling in (D, H) so every level
// keeps the 128-voxel W lines the convolution tiles on, and skip
// concatenation.  It is trained on the GPU by its own kernels: forward,
// data gradients through the same tensor-core convolution with flipped and
// transposed weights (ReLU masks fused in its epilogue), weight gradients
// on the tensor cores too (implicit GEMM over voxels, csrc/conv.cu, partial
// sums added in a fixed order, so training is bit-reproducible), and Adam
// on FP32 master weights.  Loss: the fraction of
// the error's energy that one optimal step along M(r) leaves, for the
// residual / error pairs (r, e) the plain solver's iterates give.
#include "hp_common.cuh"
#include "tc_conv.cuh"

#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <atomic>
#include <vector>

namespace hp {
namespace pc {

enum Layer { E1A, E1B, E2A, E2B, E3A, E3B, D2A, D2B, D1A, D1B, OUT, NL };
static const int LCIN[NL] = {16, 16, 16, 32, 32, 64, 96, 32, 48, 16, 16};
static const int LCOUT[NL] = {16, 16, 32, 32, 64, 64, 32, 32, 16, 16, 1};
static const int LLEV[NL] = {1, 1, 2, 2, 3, 3, 2, 2, 1, 1, 1};

__host__ __device__ inline int padc(int c) { return c < 16 ? 16 : c; }

constexpr int TB = 256;

struct Dims {
  int D, H, W;            // network level dims
  __host__ __device__ int64_t n() const { return (int64_t)D * H * W; }
};

// ------------------------------------------------------------------ kernels

// Packs FP32 master weights w[co][ci][27] into the forward operand
// [27][ci/8][coP][8] and the data-gradient operand [27][coP/8][ci][8]
// (spatially flipped, channels transposed); padded channels are zero.
__global__ void pack_kernel(const float* __restrict__ w, int cin, int cout,
                            __nv_bfloat16* __restrict__ wp, __nv_bfloat16* __restrict__ wpt) {
  const int coP = padc(cout);
  const int64_t n = (int64_t)27 * cin * coP;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    // forward: q = ((t * cin/8 + g) * coP + co) * 8 + j, ci = 8 g + j
    {
      const int j = q % 8, co = (q / 8) % coP, g = (q / (8 * coP)) % (cin / 8),
                t = (int)(q / ((int64_t)8 * coP * (cin / 8)));
      const int ci = 8 * g + j;
      const float v = co < cout ? w[((int64_t)co * cin + ci) * 27 + t] : 0.0f;
      wp[q] = __float2bfloat16(v);
    }
    // data gradient: q = ((t * coP/8 + g) * cin + ci) * 8 + j, co = 8 g + j
    {
      const int j = q % 8, ci = (q / 8) % cin, g = (q / (8 * cin)) % (coP / 8),
                t = (int)(q / ((int64_t)8 * cin * (coP / 8)));
      const int co = 8 * g + j;
      const float v = co < cout ? w[((int64_t)co * cin + ci) * 27 + (26 - t)] : 0.0f;
      wpt[q] = __float2bfloat16(v);
    }
  }
}

struct FeatArgs {
  int pj, pk;                 // padded fine dims j, k
  int64_t pin;                // padded fine index of the pinned voxel
  const uint8_t* label;       // padded fine labels
  const float* invd;          // padded fine inverse diagonal
  const float* r;             // padded fine residual
  Dims c;                     // coarse dims
};

__device__ __forceinline__ int64_t fine_of(const FeatArgs& a, int d, int h, int w, int q) {
  const int fi = 2 * d + ((q >> 2) & 1) + 1, fj = 2 * h + ((q >> 1) & 1) + 1,
            fk = 2 * w + (q & 1) + 1;
  return ((int64_t)fi * a.pj + fj) * a.pk + fk;
}

// raw[c] = mean over the 8 children of invd * r; partial sum of raw^2
__global__ void __launch_bounds__(TB) feat_raw_kernel(FeatArgs a, float* __restrict__ raw,
                                                     double* __restrict__ part) {
  double acc = 0.0;
  const int64_t n = a.c.n();
  for (int64_t c = blockIdx.x * (int64_t)TB + threadIdx.x; c < n; c += (int64_t)gridDim.x * TB) {
    const int w = c % a.c.W, h = (c / a.c.W) % a.c.H, d = (int)(c / ((int64_t)a.c.W * a.c.H));
    float s = 0.0f;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int64_t g = fine_of(a, d, h, w, q);
      if (a.label[g] != 0 && g != a.pin) s += a.invd[g] * a.r[g];
    }
    s *= 0.125f;
    raw[c] = s;
    acc += (double)s * s;
  }
  __shared__ double sh[TB];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int st = TB / 2; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st) sh[threadIdx.x] += sh[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// scale s = sqrt(mean raw^2) (single block), stored as float
__global__ void scale_kernel(const double* part, int nparts, int64_t n, float* scale) {
  __shared__ double sh[TB];
  double a = 0.0;
  for (int q = threadIdx.x; q < nparts; q += TB) a += part[q];
  sh[threadIdx.x] = a;
  __syncthreads();
  for (int st = TB / 2; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st) sh[threadIdx.x] += sh[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double rms = sqrt(sh[0] / (double)(n > 0 ? n : 1));
    scale[0] = (float)(rms > 1e-30 ? rms : 1e-30);
  }
}

// feat[c][0] = raw / s, channels 1.. from the geometry tensor, channel 15
// the coarse correction zh / s_z when there is a coarse level (zh != null)
__global__ void feat_write_kernel(const float* __restrict__ raw, const __nv_bfloat16* __restrict__ geo,
                                  const float* __restrict__ scale, __nv_bfloat16* __restrict__ feat,
                                  int64_t n, const float* __restrict__ zh) {
  const float inv = 1.0f / scale[0];
  const float invz = zh ? 1.0f / scale[1] : 0.0f;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    __align__(16) __nv_bfloat16 v[16];
    *(uint4*)&v[0] = ((const uint4*)(geo + c * 16))[0];
    *(uint4*)&v[8] = ((const uint4*)(geo + c * 16))[1];
    v[0] = __float2bfloat16(raw[c] * inv);
    if (zh) v[15] = __float2bfloat16(zh[c] * invz);
    ((uint4*)(feat + c * 16))[0] = *(uint4*)&v[0];
    ((uint4*)(feat + c * 16))[1] = *(uint4*)&v[8];
  }
}

// 2 x 2 average pooling over (D, H): out dims (D/2, H/2, W)
__global__ void pool_kernel(const __nv_bfloat16* __restrict__ in, __nv_bfloat16* __restrict__ out,
                            Dims o, int C) {
  const int64_t n = o.n() * C;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int c = q % C;
    const int64_t v = q / C;
    const int w = v % o.W, h = (v / o.W) % o.H, d = (int)(v / ((int64_t)o.W * o.H));
    const int Hi = 2 * o.H;
    float s = 0.0f;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b)
        s += __bfloat162float(in[((((int64_t)(2 * d + a) * Hi + 2 * h + b) * o.W) + w) * C + c]);
    out[q] = __float2bfloat16(0.25f * s);
  }
}

// backward of pooling: gin (fine) += 0.25 * gout (coarse)
__global__ void pool_back_kernel(const __nv_bfloat16* __restrict__ gout, __nv_bfloat16* __restrict__ gin,
                                 Dims f, int C) {
  const int64_t n = f.n() * C;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int c = q % C;
    const int64_t v = q / C;
    const int w = v % f.W, h = (v / f.W) % f.H, d = (int)(v / ((int64_t)f.W * f.H));
    const int64_t vc = ((int64_t)(d / 2) * (f.H / 2) + h / 2) * f.W + w;
    gin[q] = __float2bfloat16(__bfloat162float(gin[q]) + 0.25f * __bfloat162float(gout[vc * C + c]));
  }
}

// out (fine, C1 + C2 channels) = [nearest-upsampled coarse (C1) | skip (C2)]
__global__ void upcat_kernel(const __nv_bfloat16* __restrict__ coarse, const __nv_bfloat16* __restrict__ skip,
                             __nv_bfloat16* __restrict__ out, Dims f, int C1, int C2) {
  const int C = C1 + C2;
  const int64_t n = f.n() * (C / 8);
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int g = q % (C / 8);
    const int64_t v = q / (C / 8);
    const int w = v % f.W, h = (v / f.W) % f.H, d = (int)(v / ((int64_t)f.W * f.H));
    uint4 val;
    if (g * 8 < C1) {
      const int64_t vc = ((int64_t)(d / 2) * (f.H / 2) + h / 2) * f.W + w;
      val = *(const uint4*)(coarse + vc * C1 + g * 8);
    } else {
      val = *(const uint4*)(skip + v * C2 + (g * 8 - C1));
    }
    *(uint4*)(out + v * C + g * 8) = val;
  }
}

// backward of upcat: gcoarse = sum of the 4 fine children's first C1
// channels, gskip = remaining channels (overwrites both)
__global__ void upcat_back_kernel(const __nv_bfloat16* __restrict__ gu, __nv_bfloat16* __restrict__ gcoarse,
                                  __nv_bfloat16* __restrict__ gskip, Dims f, int C1, int C2) {
  const int C = C1 + C2;
  const Dims c{f.D / 2, f.H / 2, f.W};
  const int64_t nc = c.n() * C1;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nc;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int ch = q % C1;
    const int64_t v = q / C1;
    const int w = v % c.W, h = (v / c.W) % c.H, d = (int)(v / ((int64_t)c.W * c.H));
    float s = 0.0f;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b)
        s += __bfloat162float(gu[((((int64_t)(2 * d + a) * f.H + 2 * h + b) * f.W) + w) * C + ch]);
    gcoarse[q] = __float2bfloat16(s);
  }
  const int64_t nf = f.n() * C2;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nf;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int ch = q % C2;
    const int64_t v = q / C2;
    gskip[q] = gu[v * C + C1 + ch];
  }
}

// g = g * (a > 0) (ReLU backward on a stored activation)
__global__ void relu_mask_kernel(__nv_bfloat16* __restrict__ g, const __nv_bfloat16* __restrict__ a, int64_t n) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x)
    if (!(__bfloat162float(a[q]) > 0.0f)) g[q] = __float2bfloat16(0.0f);
}

// Coarse level: per aggregate the sum of r over its active, unpinned cells.
struct CoarseArgs {
  int ni, nj, nk, pj, pk, ag, ag_shift, nbj, nbk, nc;
  int64_t pin;
  const uint8_t* label;
  const int32_t* c_box;   // nc aggregate boxes
  const int32_t* box2c;   // per box: coarse index or -1
  const float* ainv;      // nc x nc, row-major
  double* rc;
  float* zc;
};

// aggregate edge lengths are powers of two: shifts instead of divisions
__device__ __forceinline__ int coarse_of(const CoarseArgs& c, int i, int j, int k) {
  const int sh = c.ag_shift;
  return c.box2c[((i >> sh) * c.nbj + (j >> sh)) * c.nbk + (k >> sh)];
}

__global__ void __launch_bounds__(TB) coarse_restrict_kernel(CoarseArgs c, const float* __restrict__ r) {
  const int I = blockIdx.x;
  const int b = c.c_box[I];
  const int bk = b % c.nbk, bj = (b / c.nbk) % c.nbj, bi = b / (c.nbk * c.nbj);
  const int sh = c.ag_shift, m = c.ag - 1;
  const int n = 1 << (3 * sh);
  double acc = 0.0;
  for (int t = threadIdx.x; t < n; t += TB) {
    const int i = (bi << sh) + (t >> (2 * sh)), j = (bj << sh) + ((t >> sh) & m),
              k = (bk << sh) + (t & m);
    if (i >= c.ni || j >= c.nj || k >= c.nk) continue;
    const int64_t g = ((int64_t)(i + 1) * c.pj + (j + 1)) * c.pk + (k + 1);
    if (c.label[g] != 0 && g != c.pin) acc += (double)r[g];
  }
  __shared__ double red[TB];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int st = TB / 2; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) c.rc[I] = red[0];
}

// zc = A_c^-1 rc, one warp per row
__global__ void __launch_bounds__(TB) coarse_matvec_kernel(CoarseArgs c) {
  const int row = blockIdx.x * (TB / 32) + threadIdx.x / 32, lane = threadIdx.x % 32;
  if (row >= c.nc) return;
  const float* a = c.ainv + (int64_t)row * c.nc;
  float acc = 0.0f;
  for (int q = lane; q < c.nc; q += 32) acc += a[q] * (float)c.rc[q];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) c.zc[row] = acc;
}

// zh[c] = coarse correction of the aggregate holding network cell c (its 8
// fine children share one aggregate, ag being even); partial sums of zh^2
__global__ void __launch_bounds__(TB) coarse_feat_kernel(CoarseArgs c, Dims cd, float* __restrict__ zh,
                                                         double* __restrict__ part) {
  double acc = 0.0;
  const int64_t n = cd.n();
  for (int64_t q = blockIdx.x * (int64_t)TB + threadIdx.x; q < n; q += (int64_t)gridDim.x * TB) {
    const int w = q % cd.W, h = (q / cd.W) % cd.H, d = (int)(q / ((int64_t)cd.W * cd.H));
    const int I = coarse_of(c, 2 * d, 2 * h, 2 * w);
    const float v = I >= 0 ? c.zc[I] : 0.0f;
    zh[q] = v;
    acc += (double)v * v;
  }
  __shared__ double sh[TB];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int st = TB / 2; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st) sh[threadIdx.x] += sh[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

struct ProlongArgs {
  CoarseArgs c;
  int pj, pk;
  int64_t ng, pin;
  const uint8_t* label;
  const float* invd;
  const float* r;
  const float* y;       // coarse FP32 output
  const float* scale;
  float omega;
  Dims cd;
  int use_net;
};

// z = omega * invd * r + s * y[parent] + zc[aggregate] on active fine cells
// (0 elsewhere); one block per padded (i, j) row, threads along k, so the
// coordinates come from the launch shape instead of divisions.
__global__ void __launch_bounds__(TB) prolong_kernel(ProlongArgs a, float* __restrict__ z) {
  const float s = a.use_net ? a.scale[2] : 0.0f;
  const int i = blockIdx.y, j = blockIdx.x;
  const int64_t row = ((int64_t)i * a.pj + j) * a.pk;
  const bool inner = i > 0 && j > 0 && j < a.pj - 1 && i < (int)(a.ng / ((int64_t)a.pj * a.pk)) - 1;
  for (int k = threadIdx.x; k < a.pk; k += TB) {
    const int64_t g = row + k;
    float v = 0.0f;
    if (inner && a.label[g] != 0 && g != a.pin) {
      v = a.omega * a.invd[g] * a.r[g];
      const int ui = i - 1, uj = j - 1, uk = k - 1;
      if (a.use_net) v += s * a.y[((int64_t)(ui >> 1) * a.cd.H + (uj >> 1)) * a.cd.W + (uk >> 1)];
      if (a.c.nc > 0) v += a.c.zc[coarse_of(a.c, ui, uj, uk)];
    }
    z[g] = v;
  }
}

// Training loss: how well one optimal step along z = M(r) reduces the
// energy of the error e (A e = r):
//   L = 1 - (r.z)^2 / ((z.A z) (r.e)),   dL/dz = 2 (r.z) / ((z.A z)(r.e)) ((r.z)/(z.A z) A z - r)
// which is invariant to the scale of M and weighs error components by their
// energy, as CG does.  The network output enters z as s_out * y[parent].
struct EnergyArgs {
  int pj, pk;
  int64_t ng, pin;
  const uint8_t* label;
  const float* T32;     // 16 x 16 face conductances
  const float* r;
  const float* e;
  const float* z;
  float* az;
};

// az = A z on unknown cells; block partials of r.z, z.A z, r.e
__global__ void __launch_bounds__(TB) energy_dots_kernel(EnergyArgs a, double* __restrict__ part) {
  __shared__ float T[HP_MAX_MATERIALS * HP_MAX_MATERIALS];
  for (int q = threadIdx.x; q < HP_MAX_MATERIALS * HP_MAX_MATERIALS; q += TB) T[q] = a.T32[q];
  __syncthreads();
  const int64_t SJ = a.pk, SI = (int64_t)a.pj * a.pk;
  double acc[3] = {0.0, 0.0, 0.0};
  for (int64_t g = blockIdx.x * (int64_t)TB + threadIdx.x; g < a.ng; g += (int64_t)gridDim.x * TB) {
    const int l = a.label[g];
    if (l == 0 || g == a.pin) continue;
    const float zg = a.z[g];
    const int64_t nb[6] = {g + SI, g - SI, g + SJ, g - SJ, g + 1, g - 1};
    float q = 0.0f;
#pragma unroll
    for (int f = 0; f < 6; ++f) q += T[l * HP_MAX_MATERIALS + a.label[nb[f]]] * (zg - a.z[nb[f]]);
    a.az[g] = q;
    const double rg = a.r[g];
    acc[0] += rg * zg;
    acc[1] += (double)zg * q;
    acc[2] += rg * a.e[g];
  }
  __shared__ double sh[3][TB];
#pragma unroll
  for (int k = 0; k < 3; ++k) sh[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int st = TB / 2; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st)
#pragma unroll
      for (int k = 0; k < 3; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < 3; ++k) part[3 * blockIdx.x + k] = sh[k][0];
}

__global__ void sum3_kernel(const double* part, int nparts, double* out) {
  __shared__ double sh[3][TB];
  double a[3] = {0.0, 0.0, 0.0};
  for (int q = threadIdx.x; q < nparts; q += TB)
#pragma unroll
    for (int k = 0; k < 3; ++k) a[k] += part[3 * q + k];
#pragma unroll
  for (int k = 0; k < 3; ++k) sh[k][threadIdx.x] = a[k];
  __syncthreads();
  for (int st = TB / 2; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st)
#pragma unroll
      for (int k = 0; k < 3; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < 3; ++k) out[k] = sh[k][0];
}

// dL/d(net output) into channel 0 of a 16-channel BF16 gradient tensor
// (other channels zero); the loss value into *loss
__global__ void __launch_bounds__(TB) energy_grad_kernel(EnergyArgs a, Dims cd, const double* dots,
                                                         const float* scale,
                                                         __nv_bfloat16* __restrict__ gout,
                                                         double* loss) {
  const double rz = dots[0], zaz = fmax(dots[1], 1e-300), re = dots[2];
  const double G = 2.0 * rz / (zaz * re), ratio = rz / zaz;
  const float s = scale[2];
  const int64_t n = cd.n();
  for (int64_t c = blockIdx.x * (int64_t)TB + threadIdx.x; c < n; c += (int64_t)gridDim.x * TB) {
    const int w = c % cd.W, h = (c / cd.W) % cd.H, d = (int)(c / ((int64_t)cd.W * cd.H));
    double g = 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int fi = 2 * d + ((q >> 2) & 1) + 1, fj = 2 * h + ((q >> 1) & 1) + 1,
                fk = 2 * w + (q & 1) + 1;
      const int64_t fg = ((int64_t)fi * a.pj + fj) * a.pk + fk;
      if (a.label[fg] != 0 && fg != a.pin) g += G * (ratio * a.az[fg] - (double)a.r[fg]);
    }
    __align__(16) __nv_bfloat16 o[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) o[q] = __float2bfloat16(0.0f);
    o[0] = __float2bfloat16((float)(g * s));
    ((uint4*)(gout + c * 16))[0] = *(uint4*)&o[0];
    ((uint4*)(gout + c * 16))[1] = *(uint4*)&o[8];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) loss[0] = 1.0 - rz * rz / (zaz * re);
}

// Adam on the flat parameter vector
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int64_t n, float lr, float b1, float b2, float eps,
                            float c1, float c2) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x) {
    const float gq = g[q];
    const float mq = b1 * m[q] + (1.0f - b1) * gq;
    const float vq = b2 * v[q] + (1.0f - b2) * gq * gq;
    m[q] = mq;
    v[q] = vq;
    p[q] -= lr * (mq / c1) / (sqrtf(vq / c2) + eps);
  }
}

}  // namespace pc
}  // namespace hp

using namespace hp;
using namespace hp::pc;

struct HpPrecond {
  uint64_t serial;           // unique for the process (handles may reuse an address)
  int ni, nj, nk;            // fine (unpadded) torso dims
  int pj, pk;
  int64_t ng, pin;
  Dims L[4];                 // L[1..3] network levels
  float omega;
  const uint8_t* label;      // borrowed (torso handle's padded labels) or owned
  std::vector<void*> allocs;
  // parameters: flat FP32 [all layers: w then b]
  int64_t n_par;
  float* par;
  float* grad;
  float* adam_m;
  float* adam_v;
  int64_t off_w[NL], off_b[NL];
  __nv_bfloat16* wp[NL];
  __nv_bfloat16* wpt[NL];
  float* zero_bias;          // 96 zeros
  float* wg_work;            // weight-gradient partial sums (largest layer)
  int64_t wg_bytes;
  // activations
  __nv_bfloat16 *geo, *feat, *e1a, *e1b, *p1, *e2a, *e2b, *p2, *e3a, *e3b, *u2, *d2a, *d2b, *u1,
      *d1a, *d1b;
  float* y;
  float* raw;
  float* scale;
  float* zh;                 // coarse correction on the network grid
  // gradients
  __nv_bfloat16 *gout, *g_d1b, *g_d1a, *g_u1, *g_d2b, *g_e1b, *g_d2a, *g_u2, *g_e3b, *g_e2b,
      *g_e3a, *g_p2, *g_e2a, *g_p1, *g_e1a;
  double* part;
  double* dots;              // r.z, z.A z, r.e of the energy loss
  double* loss;
  float* zbuf;               // M(r) on the fine grid (training)
  float* az;                 // A M(r)
  float* T32;                // face conductances (device, 16 x 16)
  int* err;
  int64_t step;
  int nblk;
  // coarse level (nc = 0: none)
  int ag, nbi, nbj, nbk, nc;
  int32_t* c_box;
  int32_t* box2c;
  float* ainv;
  double* rc;
  float* zc;
};

template <typename T>
static hp_status pal(HpPrecond* h, T** dst, size_t n) {
  hp_status st = dev_alloc(dst, n);
  if (st == HP_OK && *dst) h->allocs.push_back((void*)*dst);
  return st;
}

#define PC_TRY(x)                \
  do {                           \
    hp_status _s = (x);          \
    if (_s != HP_OK) {           \
      hp_precond_destroy(h);     \
      return _s;                 \
    }                            \
  } while (0)

extern "C" hp_status hp_precond_destroy(HpPrecond* h);

#define HP_TRY_PC(x)             \
  do {                           \
    hp_status _s = (x);          \
    if (_s != HP_OK) return _s;  \
  } while (0)

static hp_status repack(HpPrecond* h, cudaStream_t s) {
  for (int l = 0; l < NL; ++l) {
    pack_kernel<<<256, 256, 0, s>>>(h->par + h->off_w[l], LCIN[l], LCOUT[l], h->wp[l], h->wpt[l]);
  }
  HP_CUDA_TRY(cudaGetLastError());
  return HP_OK;
}

// Dense SPD inverse on the host (FP64): Cholesky A = L L^T, X = L^-1, then
// A^-1 = X^T X.  Returns false if A is not positive definite.
static bool spd_inverse(std::vector<double>& A, int n) {
  for (int j = 0; j < n; ++j) {
    double* Aj = &A[(size_t)j * n];
    double sjj = Aj[j];
    for (int k = 0; k < j; ++k) sjj -= Aj[k] * Aj[k];
    if (!(sjj > 0.0)) return false;
    const double ljj = sqrt(sjj);
    Aj[j] = ljj;
    for (int i = j + 1; i < n; ++i) {
      double* Ai = &A[(size_t)i * n];
      double sij = Ai[j];
      for (int k = 0; k < j; ++k) sij -= Ai[k] * Aj[k];
      Ai[j] = sij / ljj;
    }
  }
  // X = L^-1 (lower), stored transposed as U = X^T (upper, row-major)
  std::vector<double> U((size_t)n * n, 0.0), x(n);
  for (int j = 0; j < n; ++j) {
    for (int i = 0; i < j; ++i) x[i] = 0.0;
    for (int i = j; i < n; ++i) {
      const double* Li = &A[(size_t)i * n];
      double v = i == j ? 1.0 : 0.0;
      for (int k = j; k < i; ++k) v -= Li[k] * x[k];
      x[i] = v / Li[i];
    }
    for (int i = j; i < n; ++i) U[(size_t)j * n + i] = x[i];
  }
  // A^-1[i][j] = sum_k X[k][i] X[k][j] = sum_{k >= max(i,j)} U[i][k] U[j][k]
  for (int i = 0; i < n; ++i)
    for (int j = 0; j <= i; ++j) {
      const double* Ui = &U[(size_t)i * n];
      const double* Uj = &U[(size_t)j * n];
      double v = 0.0;
      for (int k = i; k < n; ++k) v += Ui[k] * Uj[k];
      A[(size_t)i * n + j] = v;
      A[(size_t)j * n + i] = v;
    }
  return true;
}

// Aggregates of ag^3 voxels (ag doubling from 4 until at most HP_PC_MAX_COARSE
// aggregates hold an active unpinned voxel, unless d->coarse_agg fixes it),
// the Galerkin operator A_c = Q^T A Q of the torso stiffness (harmonic-mean
// face conductance / h^2, air faces skipped, the pinned voxel eliminated) and
// its inverse.
static hp_status coarse_setup(HpPrecond* h, const HpPrecondDesc* d, cudaStream_t s) {
  HP_REQUIRE(d->sigma && d->h_m > 0.0, "hp_precond_create: the coarse level needs sigma and h_m");
  const int ni = d->ni, nj = d->nj, nk = d->nk;
  const int64_t pin = d->pin_cell;
  const int pjj = nj + 2, pkk = nk + 2;
  const int pin_i = pin >= 0 ? (int)(pin / ((int64_t)pjj * pkk)) - 1 : -1;
  const int pin_j = pin >= 0 ? (int)((pin / pkk) % pjj) - 1 : -1;
  const int pin_k = pin >= 0 ? (int)(pin % pkk) - 1 : -1;
  auto lab = [&](int i, int j, int k) -> int {
    if (i < 0 || j < 0 || k < 0 || i >= ni || j >= nj || k >= nk) return 0;
    return d->label[((int64_t)i * nj + j) * nk + k];
  };
  auto unknown = [&](int i, int j, int k) {
    return lab(i, j, k) != 0 && !(i == pin_i && j == pin_j && k == pin_k);
  };
  HP_REQUIRE(d->coarse_agg <= 0 || (d->coarse_agg & (d->coarse_agg - 1)) == 0,
             "hp_precond_create: coarse_agg must be a power of two");
  int ag = d->coarse_agg > 0 ? d->coarse_agg : 4;
  std::vector<int32_t> box2c, c_box;
  int nbi = 0, nbj = 0, nbk = 0;
  while (true) {
    nbi = (ni + ag - 1) / ag; nbj = (nj + ag - 1) / ag; nbk = (nk + ag - 1) / ag;
    box2c.assign((size_t)nbi * nbj * nbk, -1);
    c_box.clear();
    for (int i = 0; i < ni; ++i)
      for (int j = 0; j < nj; ++j)
        for (int k = 0; k < nk; ++k)
          if (unknown(i, j, k)) {
            const int b = ((i / ag) * nbj + j / ag) * nbk + k / ag;
            if (box2c[b] < 0) box2c[b] = 0;
          }
    for (size_t b = 0; b < box2c.size(); ++b)
      if (box2c[b] == 0) { box2c[b] = (int32_t)c_box.size(); c_box.push_back((int32_t)b); }
    if ((int)c_box.size() <= HP_PC_MAX_COARSE || d->coarse_agg > 0) break;
    ag *= 2;
  }
  const int nc = (int)c_box.size();
  HP_REQUIRE(nc <= HP_PC_MAX_COARSE, "hp_precond_create: %d coarse unknowns exceed %d", nc,
             HP_PC_MAX_COARSE);
  if (nc == 0) return HP_OK;
  double T64[HP_MAX_MATERIALS * HP_MAX_MATERIALS] = {0};
  const double h2 = d->h_m * d->h_m;
  for (int u = 1; u < d->n_materials; ++u)
    for (int v = 1; v < d->n_materials; ++v) {
      const double su = d->sigma[u], sv = d->sigma[v];
      if (su + sv >= 1e-30) T64[u * HP_MAX_MATERIALS + v] = (2.0 * su * sv) / (su + sv) / h2;
    }
  std::vector<double> Ac((size_t)nc * nc, 0.0);
  auto cid = [&](int i, int j, int k) { return box2c[((i / ag) * nbj + j / ag) * nbk + k / ag]; };
  const int off[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
  for (int i = 0; i < ni; ++i)
    for (int j = 0; j < nj; ++j)
      for (int k = 0; k < nk; ++k) {
        if (!unknown(i, j, k)) continue;
        const int I = cid(i, j, k), l = lab(i, j, k);
        for (int f = 0; f < 6; ++f) {
          const int a = i + off[f][0], b = j + off[f][1], c = k + off[f][2];
          const double t = T64[l * HP_MAX_MATERIALS + lab(a, b, c)];
          if (t == 0.0) continue;
          Ac[(size_t)I * nc + I] += t;
          if (unknown(a, b, c)) Ac[(size_t)I * nc + cid(a, b, c)] -= t;
        }
      }
  HP_REQUIRE(spd_inverse(Ac, nc), "hp_precond_create: coarse operator is not positive definite "
             "(torso not connected to the pinned voxel?)");
  std::vector<float> a32(Ac.begin(), Ac.end());
  h->ag = ag; h->nbi = nbi; h->nbj = nbj; h->nbk = nbk; h->nc = nc;
  HP_TRY_PC(pal(h, &h->c_box, nc));
  HP_TRY_PC(pal(h, &h->box2c, box2c.size()));
  HP_TRY_PC(pal(h, &h->ainv, (size_t)nc * nc));
  HP_TRY_PC(pal(h, &h->rc, nc));
  HP_TRY_PC(pal(h, &h->zc, nc));
  HP_CUDA_TRY(cudaMemcpyAsync(h->c_box, c_box.data(), nc * 4, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemcpyAsync(h->box2c, box2c.data(), box2c.size() * 4, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemcpyAsync(h->ainv, a32.data(), a32.size() * 4, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));  // host vectors are temporaries
  return HP_OK;
}

extern "C" hp_status hp_precond_create(const HpPrecondDesc* d, HpPrecond** out, void* stream) {
  HP_REQUIRE(d && out, "hp_precond_create: null argument");
  *out = nullptr;
  HP_REQUIRE(d->ni % 8 == 0 && d->nj % 8 == 0 && d->nk % 256 == 0,
             "hp_precond_create: torso dims (%d,%d,%d) must be multiples of (8,8,256)", d->ni,
             d->nj, d->nk);
  HP_REQUIRE(d->label && d->n_materials >= 1 && d->n_materials <= HP_MAX_MATERIALS,
             "hp_precond_create: bad labels");
  HP_REQUIRE(d->sigma && d->h_m > 0.0, "hp_precond_create: sigma and h_m are required");
  cudaStream_t s = (cudaStream_t)stream;
  HpPrecond* h = new HpPrecond();
  static std::atomic<uint64_t> next_serial{0};
  h->serial = ++next_serial;
  h->ni = d->ni; h->nj = d->nj; h->nk = d->nk;
  h->pj = d->nj + 2; h->pk = d->nk + 2;
  h->ng = (int64_t)(d->ni + 2) * h->pj * h->pk;
  h->pin = d->pin_cell;
  h->omega = d->omega;
  h->L[1] = Dims{d->ni / 2, d->nj / 2, d->nk / 2};
  h->L[2] = Dims{d->ni / 4, d->nj / 4, d->nk / 2};
  h->L[3] = Dims{d->ni / 8, d->nj / 8, d->nk / 2};
  h->step = 0;
  int nsm = 148;
  {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  }
  h->nblk = nsm * 8;
  // parameters
  int64_t o = 0;
  for (int l = 0; l < NL; ++l) {
    h->off_w[l] = o;
    o += (int64_t)LCOUT[l] * LCIN[l] * 27;
    h->off_b[l] = o;
    o += LCOUT[l];
  }
  h->n_par = o;
  PC_TRY(pal(h, &h->par, o));
  PC_TRY(pal(h, &h->grad, o));
  PC_TRY(pal(h, &h->adam_m, o));
  PC_TRY(pal(h, &h->adam_v, o));
  {
    // He-normal initial weights, zero biases (seeded, host-generated)
    std::vector<float> w0(o, 0.0f);
    uint64_t st = d->seed * 6364136223846793005ull + 1442695040888963407ull;
    auto unif = [&]() {
      st = st * 6364136223846793005ull + 1442695040888963407ull;
      return ((st >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    };
    for (int l = 0; l < NL; ++l) {
      const double sd = sqrt(2.0 / (27.0 * LCIN[l])) * (l == OUT ? 0.1 : 1.0);
      for (int64_t q = 0; q < (int64_t)LCOUT[l] * LCIN[l] * 27; ++q) {
        const double u1 = unif(), u2 = unif();
        w0[h->off_w[l] + q] = (float)(sd * sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2));
      }
    }
    if (d->init_params) std::copy(d->init_params, d->init_params + o, w0.begin());
    HP_CUDA_TRY(cudaMemcpyAsync(h->par, w0.data(), o * 4, cudaMemcpyHostToDevice, s));
    HP_CUDA_TRY(cudaMemsetAsync(h->adam_m, 0, o * 4, s));
    HP_CUDA_TRY(cudaMemsetAsync(h->adam_v, 0, o * 4, s));
    HP_CUDA_TRY(cudaStreamSynchronize(s));
  }
  for (int l = 0; l < NL; ++l) {
    const size_t np = (size_t)27 * LCIN[l] * padc(LCOUT[l]);
    PC_TRY(pal(h, &h->wp[l], np));
    PC_TRY(pal(h, &h->wpt[l], np));
  }
  PC_TRY(pal(h, &h->zero_bias, 96));
  HP_CUDA_TRY(cudaMemsetAsync(h->zero_bias, 0, 96 * 4, s));
  h->wg_bytes = 0;
  for (int l = 0; l < NL; ++l) {
    const Dims dm = h->L[LLEV[l]];
    h->wg_bytes = std::max(h->wg_bytes, tc::wgrad3_workspace(dm.D, dm.H, dm.W, LCIN[l], LCOUT[l]));
  }
  PC_TRY(pal(h, &h->wg_work, (h->wg_bytes + 3) / 4));
  const int64_t n1 = h->L[1].n(), n2 = h->L[2].n(), n3 = h->L[3].n();
  PC_TRY(pal(h, &h->geo, n1 * 16));
  PC_TRY(pal(h, &h->feat, n1 * 16));
  PC_TRY(pal(h, &h->e1a, n1 * 16));
  PC_TRY(pal(h, &h->e1b, n1 * 16));
  PC_TRY(pal(h, &h->p1, n2 * 16));
  PC_TRY(pal(h, &h->e2a, n2 * 32));
  PC_TRY(pal(h, &h->e2b, n2 * 32));
  PC_TRY(pal(h, &h->p2, n3 * 32));
  PC_TRY(pal(h, &h->e3a, n3 * 64));
  PC_TRY(pal(h, &h->e3b, n3 * 64));
  PC_TRY(pal(h, &h->u2, n2 * 96));
  PC_TRY(pal(h, &h->d2a, n2 * 32));
  PC_TRY(pal(h, &h->d2b, n2 * 32));
  PC_TRY(pal(h, &h->u1, n1 * 48));
  PC_TRY(pal(h, &h->d1a, n1 * 16));
  PC_TRY(pal(h, &h->d1b, n1 * 16));
  PC_TRY(pal(h, &h->y, n1));
  PC_TRY(pal(h, &h->raw, n1));
  PC_TRY(pal(h, &h->scale, 3));  // input scale s, coarse-field scale s_z, output scale
  PC_TRY(pal(h, &h->zh, n1));
  PC_TRY(pal(h, &h->gout, n1 * 16));
  PC_TRY(pal(h, &h->g_d1b, n1 * 16));
  PC_TRY(pal(h, &h->g_d1a, n1 * 16));
  PC_TRY(pal(h, &h->g_u1, n1 * 48));
  PC_TRY(pal(h, &h->g_d2b, n2 * 32));
  PC_TRY(pal(h, &h->g_e1b, n1 * 16));
  PC_TRY(pal(h, &h->g_d2a, n2 * 32));
  PC_TRY(pal(h, &h->g_u2, n2 * 96));
  PC_TRY(pal(h, &h->g_e3b, n3 * 64));
  PC_TRY(pal(h, &h->g_e2b, n2 * 32));
  PC_TRY(pal(h, &h->g_e3a, n3 * 64));
  PC_TRY(pal(h, &h->g_p2, n3 * 32));
  PC_TRY(pal(h, &h->g_e2a, n2 * 32));
  PC_TRY(pal(h, &h->g_p1, n2 * 16));
  PC_TRY(pal(h, &h->g_e1a, n1 * 16));
  PC_TRY(pal(h, &h->part, 3 * h->nblk));
  PC_TRY(pal(h, &h->dots, 3));
  PC_TRY(pal(h, &h->zbuf, h->ng));
  PC_TRY(pal(h, &h->az, h->ng));
  PC_TRY(pal(h, &h->T32, HP_MAX_MATERIALS * HP_MAX_MATERIALS));
  {
    float T32[HP_MAX_MATERIALS * HP_MAX_MATERIALS] = {0};
    const double h2 = d->h_m * d->h_m;
    for (int u = 1; u < d->n_materials; ++u)
      for (int v = 1; v < d->n_materials; ++v) {
        const double su = d->sigma[u], sv = d->sigma[v];
        if (su + sv >= 1e-30) T32[u * HP_MAX_MATERIALS + v] = (float)((2.0 * su * sv) / (su + sv) / h2);
      }
    HP_CUDA_TRY(cudaMemcpyAsync(h->T32, T32, sizeof(T32), cudaMemcpyHostToDevice, s));
    HP_CUDA_TRY(cudaStreamSynchronize(s));
  }
  PC_TRY(pal(h, &h->loss, 1));
  PC_TRY(pal(h, &h->err, 1));
  HP_CUDA_TRY(cudaMemsetAsync(h->err, 0, 4, s));
  // geometry channels on the network grid (host): active fraction and the
  // fraction of each material among the 8 fine children
  {
    const int ni = d->ni, nj = d->nj, nk = d->nk;
    std::vector<__nv_bfloat16> geo((size_t)n1 * 16, __float2bfloat16(0.0f));
    const Dims c = h->L[1];
    for (int a = 0; a < c.D; ++a)
      for (int b = 0; b < c.H; ++b)
        for (int w = 0; w < c.W; ++w) {
          float frac[HP_MAX_MATERIALS] = {0};
          for (int q = 0; q < 8; ++q) {
            const int i = 2 * a + ((q >> 2) & 1), j = 2 * b + ((q >> 1) & 1), k = 2 * w + (q & 1);
            frac[d->label[((int64_t)i * nj + j) * nk + k]] += 0.125f;
          }
          const int64_t cc = ((int64_t)a * c.H + b) * c.W + w;
          geo[cc * 16 + 1] = __float2bfloat16(1.0f - frac[0]);
          for (int m = 1; m < d->n_materials && m < 14; ++m)  // channel 15: coarse field
            geo[cc * 16 + 1 + m] = __float2bfloat16(frac[m]);
        }
    (void)ni;
    (void)nk;
    HP_CUDA_TRY(cudaMemcpyAsync(h->geo, geo.data(), geo.size() * 2, cudaMemcpyHostToDevice, s));
    HP_CUDA_TRY(cudaStreamSynchronize(s));
  }
  h->nc = 0;
  if (d->coarse_agg >= 0) PC_TRY(coarse_setup(h, d, s));
  PC_TRY(repack(h, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  *out = h;
  return HP_OK;
}

namespace hp {
namespace pc {

static hp_status conv(HpPrecond* h, int l, const __nv_bfloat16* X, void* Y, int epi,
                      const __nv_bfloat16* mask, cudaStream_t s) {
  const Dims dm = h->L[LLEV[l]];
  return tc::conv3_launch(X, h->wp[l], h->par + h->off_b[l], Y, mask, dm.D, dm.H, dm.W, LCIN[l],
                          padc(LCOUT[l]), epi, h->err, s);
}

// data gradient of layer l: gin = conv(gpre, flipped W^T), optional mask
static hp_status dgrad(HpPrecond* h, int l, const __nv_bfloat16* gpre, __nv_bfloat16* gin,
                       const __nv_bfloat16* mask, cudaStream_t s) {
  const Dims dm = h->L[LLEV[l]];
  return tc::conv3_launch(gpre, h->wpt[l], h->zero_bias, gin, mask, dm.D, dm.H, dm.W,
                          padc(LCOUT[l]), LCIN[l], mask ? tc::EPI_MASK : tc::EPI_LINEAR, h->err, s);
}

// weight and bias gradients of layer l on the tensor cores (tc::wgrad3_launch:
// implicit GEMM over voxels, partial sums added in a fixed order)
static hp_status wgrad(HpPrecond* h, int l, const __nv_bfloat16* X, const __nv_bfloat16* G,
                       cudaStream_t s) {
  const Dims dm = h->L[LLEV[l]];
  return tc::wgrad3_launch(X, G, dm.D, dm.H, dm.W, LCIN[l], LCOUT[l], h->grad + h->off_w[l],
                           h->grad + h->off_b[l], h->wg_work, h->wg_bytes, h->err, s);
}

static int grid_for(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>(4096, (n + 255) / 256)); }

static CoarseArgs coarse_args(const HpPrecond* h, const uint8_t* label) {
  int sh = 0;
  while ((1 << sh) < h->ag) ++sh;
  return CoarseArgs{h->ni, h->nj, h->nk, h->pj, h->pk, h->ag, sh, h->nbj, h->nbk, h->nc, h->pin,
                    label, h->c_box, h->box2c, h->ainv, h->rc, h->zc};
}

// zc = A_c^-1 Q^T r (no-op without a coarse level)
static hp_status coarse_solve(HpPrecond* h, const uint8_t* label, const float* r, cudaStream_t s) {
  if (h->nc == 0) return HP_OK;
  const CoarseArgs c = coarse_args(h, label);
  coarse_restrict_kernel<<<h->nc, TB, 0, s>>>(c, r);
  coarse_matvec_kernel<<<(h->nc + TB / 32 - 1) / (TB / 32), TB, 0, s>>>(c);
  HP_CUDA_TRY(cudaGetLastError());
  return HP_OK;
}

hp_status precond_forward(HpPrecond* h, const uint8_t* label, const float* invd, const float* r,
                          cudaStream_t s) {
  FeatArgs fa{h->pj, h->pk, h->pin, label, invd, r, h->L[1]};
  const int64_t n1 = h->L[1].n();
  feat_raw_kernel<<<h->nblk, TB, 0, s>>>(fa, h->raw, h->part);
  scale_kernel<<<1, TB, 0, s>>>(h->part, h->nblk, n1, h->scale);
  if (h->nc > 0) {
    // the network also sees the coarse correction; its output is scaled like
    // that field (the error it refines), else like the input
    coarse_feat_kernel<<<h->nblk, TB, 0, s>>>(coarse_args(h, label), h->L[1], h->zh, h->part);
    scale_kernel<<<1, TB, 0, s>>>(h->part, h->nblk, n1, h->scale + 1);
    HP_CUDA_TRY(cudaMemcpyAsync(h->scale + 2, h->scale + 1, 4, cudaMemcpyDeviceToDevice, s));
  } else {
    HP_CUDA_TRY(cudaMemcpyAsync(h->scale + 2, h->scale, 4, cudaMemcpyDeviceToDevice, s));
  }
  feat_write_kernel<<<grid_for(n1), 256, 0, s>>>(h->raw, h->geo, h->scale, h->feat, n1,
                                                 h->nc > 0 ? h->zh : nullptr);
  HP_CUDA_TRY(cudaGetLastError());
  hp_status st;
#define FW(x) do { st = (x); if (st != HP_OK) return st; } while (0)
  FW(conv(h, E1A, h->feat, h->e1a, tc::EPI_RELU, nullptr, s));
  FW(conv(h, E1B, h->e1a, h->e1b, tc::EPI_RELU, nullptr, s));
  pool_kernel<<<grid_for(h->L[2].n() * 16), 256, 0, s>>>(h->e1b, h->p1, h->L[2], 16);
  FW(conv(h, E2A, h->p1, h->e2a, tc::EPI_RELU, nullptr, s));
  FW(conv(h, E2B, h->e2a, h->e2b, tc::EPI_RELU, nullptr, s));
  pool_kernel<<<grid_for(h->L[3].n() * 32), 256, 0, s>>>(h->e2b, h->p2, h->L[3], 32);
  FW(conv(h, E3A, h->p2, h->e3a, tc::EPI_RELU, nullptr, s));
  FW(conv(h, E3B, h->e3a, h->e3b, tc::EPI_RELU, nullptr, s));
  upcat_kernel<<<grid_for(h->L[2].n() * 12), 256, 0, s>>>(h->e3b, h->e2b, h->u2, h->L[2], 64, 32);
  FW(conv(h, D2A, h->u2, h->d2a, tc::EPI_RELU, nullptr, s));
  FW(conv(h, D2B, h->d2a, h->d2b, tc::EPI_RELU, nullptr, s));
  upcat_kernel<<<grid_for(h->L[1].n() * 6), 256, 0, s>>>(h->d2b, h->e1b, h->u1, h->L[1], 32, 16);
  FW(conv(h, D1A, h->u1, h->d1a, tc::EPI_RELU, nullptr, s));
  FW(conv(h, D1B, h->d1a, h->d1b, tc::EPI_RELU, nullptr, s));
  FW(conv(h, OUT, h->d1b, h->y, tc::EPI_F32_C0, nullptr, s));
#undef FW
  HP_CUDA_TRY(cudaGetLastError());
  return HP_OK;
}

uint64_t precond_serial(const HpPrecond* h) { return h->serial; }

hp_status precond_apply(HpPrecond* h, const uint8_t* label, const float* invd, const float* r,
                        float* z, int use_net, cudaStream_t s) {
  hp_status cst = coarse_solve(h, label, r, s);
  if (cst != HP_OK) return cst;
  if (use_net) {
    hp_status st = precond_forward(h, label, invd, r, s);
    if (st != HP_OK) return st;
  }
  ProlongArgs pa{coarse_args(h, label), h->pj, h->pk, h->ng, h->pin, label, invd, r, h->y,
                 h->scale, h->omega, h->L[1], use_net};
  prolong_kernel<<<dim3(h->pj, (unsigned)(h->ng / ((int64_t)h->pj * h->pk))), TB, 0, s>>>(pa, z);
  HP_CUDA_TRY(cudaGetLastError());
  return HP_OK;
}

}  // namespace pc
}  // namespace hp

extern "C" hp_status hp_precond_apply(HpPrecond* h, const uint8_t* label, const float* invd,
                                      const float* r, float* z, int32_t use_net, void* stream) {
  HP_REQUIRE(h && label && invd && r && z, "hp_precond_apply: null argument");
  return hp::pc::precond_apply(h, label, invd, r, z, use_net, (cudaStream_t)stream);
}

extern "C" hp_status hp_precond_train_step(HpPrecond* h, const uint8_t* label, const float* invd,
                                           const float* r, const float* e, float lr,
                                           float* loss_out, void* stream) {
  HP_REQUIRE(h && label && invd && r && e, "hp_precond_train_step: null argument");
  cudaStream_t s = (cudaStream_t)stream;
  hp_status st = coarse_solve(h, label, r, s);
  if (st != HP_OK) return st;
  st = precond_forward(h, label, invd, r, s);
  if (st != HP_OK) return st;
  const Dims L1 = h->L[1], L2 = h->L[2], L3 = h->L[3];
  const int64_t n1 = L1.n(), n2 = L2.n(), n3 = L3.n();
  ProlongArgs pa{coarse_args(h, label), h->pj, h->pk, h->ng, h->pin, label, invd, r, h->y,
                 h->scale, h->omega, h->L[1], 1};
  prolong_kernel<<<dim3(h->pj, (unsigned)(h->ng / ((int64_t)h->pj * h->pk))), TB, 0, s>>>(pa, h->zbuf);
  EnergyArgs ea{h->pj, h->pk, h->ng, h->pin, label, h->T32, r, e, h->zbuf, h->az};
  energy_dots_kernel<<<h->nblk, TB, 0, s>>>(ea, h->part);
  sum3_kernel<<<1, TB, 0, s>>>(h->part, h->nblk, h->dots);
  energy_grad_kernel<<<h->nblk, TB, 0, s>>>(ea, L1, h->dots, h->scale, h->gout, h->loss);
  HP_CUDA_TRY(cudaMemsetAsync(h->grad, 0, h->n_par * 4, s));
#define BW(x) do { st = (x); if (st != HP_OK) return st; } while (0)
  // OUT (linear, 16 -> 1 padded to 16)
  BW(wgrad(h, OUT, h->d1b, h->gout, s));
  BW(dgrad(h, OUT, h->gout, h->g_d1b, h->d1b, s));          // -> dpre of D1B
  BW(wgrad(h, D1B, h->d1a, h->g_d1b, s));
  BW(dgrad(h, D1B, h->g_d1b, h->g_d1a, h->d1a, s));         // -> dpre of D1A
  BW(wgrad(h, D1A, h->u1, h->g_d1a, s));
  BW(dgrad(h, D1A, h->g_d1a, h->g_u1, nullptr, s));         // d u1 (48)
  upcat_back_kernel<<<grid_for(n1 * 16), 256, 0, s>>>(h->g_u1, h->g_d2b, h->g_e1b, L1, 32, 16);
  relu_mask_kernel<<<grid_for(n2 * 32), 256, 0, s>>>(h->g_d2b, h->d2b, n2 * 32);
  BW(wgrad(h, D2B, h->d2a, h->g_d2b, s));
  BW(dgrad(h, D2B, h->g_d2b, h->g_d2a, h->d2a, s));
  BW(wgrad(h, D2A, h->u2, h->g_d2a, s));
  BW(dgrad(h, D2A, h->g_d2a, h->g_u2, nullptr, s));         // d u2 (96)
  upcat_back_kernel<<<grid_for(n2 * 64), 256, 0, s>>>(h->g_u2, h->g_e3b, h->g_e2b, L2, 64, 32);
  relu_mask_kernel<<<grid_for(n3 * 64), 256, 0, s>>>(h->g_e3b, h->e3b, n3 * 64);
  BW(wgrad(h, E3B, h->e3a, h->g_e3b, s));
  BW(dgrad(h, E3B, h->g_e3b, h->g_e3a, h->e3a, s));
  BW(wgrad(h, E3A, h->p2, h->g_e3a, s));
  BW(dgrad(h, E3A, h->g_e3a, h->g_p2, nullptr, s));
  pool_back_kernel<<<grid_for(n2 * 32), 256, 0, s>>>(h->g_p2, h->g_e2b, L2, 32);
  relu_mask_kernel<<<grid_for(n2 * 32), 256, 0, s>>>(h->g_e2b, h->e2b, n2 * 32);
  BW(wgrad(h, E2B, h->e2a, h->g_e2b, s));
  BW(dgrad(h, E2B, h->g_e2b, h->g_e2a, h->e2a, s));
  BW(wgrad(h, E2A, h->p1, h->g_e2a, s));
  BW(dgrad(h, E2A, h->g_e2a, h->g_p1, nullptr, s));
  pool_back_kernel<<<grid_for(n1 * 16), 256, 0, s>>>(h->g_p1, h->g_e1b, L1, 16);
  relu_mask_kernel<<<grid_for(n1 * 16), 256, 0, s>>>(h->g_e1b, h->e1b, n1 * 16);
  BW(wgrad(h, E1B, h->e1a, h->g_e1b, s));
  BW(dgrad(h, E1B, h->g_e1b, h->g_e1a, h->e1a, s));
  BW(wgrad(h, E1A, h->feat, h->g_e1a, s));
#undef BW
  HP_CUDA_TRY(cudaGetLastError());
  if (lr > 0.0f) {
    h->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - powf(b1, (float)h->step), c2 = 1.0f - powf(b2, (float)h->step);
    adam_kernel<<<grid_for(h->n_par), 256, 0, s>>>(h->par, h->grad, h->adam_m, h->adam_v,
                                                   h->n_par, lr, b1, b2, 1e-8f, c1, c2);
    st = repack(h, s);
    if (st != HP_OK) return st;
  }
  if (loss_out) {
    double l = 0.0;
    HP_CUDA_TRY(cudaMemcpyAsync(&l, h->loss, 8, cudaMemcpyDeviceToHost, s));
    HP_CUDA_TRY(cudaStreamSynchronize(s));
    *loss_out = (float)l;
  }
  return HP_OK;
}

extern "C" hp_status hp_precond_params(HpPrecond* h, float* host_params, float* host_grads,
                                       int64_t* n, int32_t set, void* stream) {
  HP_REQUIRE(h && n, "hp_precond_params: null argument");
  cudaStream_t s = (cudaStream_t)stream;
  *n = h->n_par;
  if (set && host_params) {
    HP_CUDA_TRY(cudaMemcpyAsync(h->par, host_params, h->n_par * 4, cudaMemcpyHostToDevice, s));
    hp_status st = repack(h, s);
    if (st != HP_OK) return st;
  } else if (host_params) {
    HP_CUDA_TRY(cudaMemcpyAsync(host_params, h->par, h->n_par * 4, cudaMemcpyDeviceToHost, s));
  }
  if (host_grads)
    HP_CUDA_TRY(cudaMemcpyAsync(host_grads, h->grad, h->n_par * 4, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  return HP_OK;
}

extern "C" hp_status hp_precond_output(HpPrecond* h, float* host_y, float* host_scale,
                                       int32_t* host_err, void* stream) {
  HP_REQUIRE(h, "hp_precond_output: null handle");
  cudaStream_t s = (cudaStream_t)stream;
  if (host_y) HP_CUDA_TRY(cudaMemcpyAsync(host_y, h->y, h->L[1].n() * 4, cudaMemcpyDeviceToHost, s));
  if (host_scale) HP_CUDA_TRY(cudaMemcpyAsync(host_scale, h->scale, 4, cudaMemcpyDeviceToHost, s));
  if (host_err) HP_CUDA_TRY(cudaMemcpyAsync(host_err, h->err, 4, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  return HP_OK;
}

extern "C" hp_status hp_precond_coarse_info(const HpPrecond* h, int32_t* agg, int32_t* n_coarse) {
  HP_REQUIRE(h, "hp_precond_coarse_info: null handle");
  if (agg) *agg = h->nc ? h->ag : 0;
  if (n_coarse) *n_coarse = h->nc;
  return HP_OK;
}

extern "C" hp_status hp_precond_destroy(HpPrecond* h) {
  if (!h) return HP_OK;
  for (void* p : h->allocs) cudaFree(p);
  delete h;
  return HP_OK;
}
