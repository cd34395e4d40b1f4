// Per-frame torso Poisson solve (ECG forward problem) for sm_100a.
//
// Replaces make_gpu_solver / solve_frame / _pcg_gpu of the reference
// (ecg/functions/compute_bspm.py:164-436) over the sharp-boundary 7-point
// operator of _assemble_stiffness (ecg/functions/build_torso_grid.py:276-397):
//   A_kk = sum_faces g_f,  A_kn = -g_f,  g_f = harm(sigma_k, sigma_n) / h^2,
// air faces skipped (Neumann), one pinned row fixed to 0.
//
// The operator is never assembled.  Conductivity is piecewise constant by
// material label, so a face conductance is a lookup in an M x M table; the
// solver keeps one byte per voxel of operator data instead of 7 CSR entries.
// Grid arrays are dense over the torso box padded by one air voxel on every
// side (no bounds tests in the stencil); k is the fastest axis, so a warp's
// accesses and its +/-k neighbours are contiguous and the +/-j, +/-i
// neighbours are rows / planes that the previous warps just brought into L2.
//
// Precision: vectors r, p, Ap and the SpMV run in FP32; the solution x and
// every dot product / norm are FP64; the convergence decision for the
// relative rule is taken on the FP64 true residual b - A x evaluated with the
// FP64 conductance table (the reference operator's own coefficients).  If the
// recursive FP32 residual claims convergence but the true residual does not,
// r is replaced by the true residual and CG restarts (residual replacement).
//
// Reductions are deterministic: each block writes its partial, the last block
// to arrive (atomic ticket after __threadfence) sums the partials in block
// order and updates the scalars.  No kernel ever waits on another block.
#include "hp_common.cuh"

#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <vector>

namespace hp {

constexpr int TB = 256;            // threads per block
// resident blocks per SM the register budgets of the iteration kernels are
// sized for (1: the compiler's choice)
#ifndef HP_AP_MINB
#define HP_AP_MINB 4  // pcg_ap: 64 registers (86.2 us per iteration on the full torso, 89.4 at 80)
#endif
#ifndef HP_K2_MINB
#define HP_K2_MINB 1
#endif
#ifndef HP_PU_MINB
#define HP_PU_MINB 1
#endif
constexpr int NPART = 4;           // partial sums per block

enum Scal : int {
  SC_RZ = 0, SC_PAP, SC_ALPHA, SC_BETA, SC_ALPHA_PREV, SC_ZZ, SC_ZMAX, SC_RR, SC_BB,
  SC_TRUE_RR, SC_SRC_MEAN, SC_STAT, SC_TOL, SC_HIST0, N_SCAL = SC_HIST0 + 8
};
enum IScal : int {
  IS_DONE = 0, IS_ITER, IS_RULE, IS_MAXIT, IS_BREAKDOWN, IS_NONFINITE, IS_STAGNANT, IS_NH,
  IS_STAG_ON, N_ISCAL
};

struct TorsoArgs {
  int64_t ng;          // padded grid cells
  int32_t pj, pk;      // padded dims j, k (i stride = pj * pk)
  const uint8_t* label;
  const float* invd;
  float* r;
  float* p0;
  float* p1;
  float* Ap;
  double* x;
  float* b;
  int64_t pin;         // padded grid index of the pinned voxel
  int64_t n_rows;
  double* scal;
  int32_t* iscal;
  double* part;        // gridDim x NPART
  unsigned int* ticket;
  // tissue lines: the k-run from the first to the last tissue cell of every
  // (i, j) line that has one (air inside a run is allowed)
  int32_t n_lines;
  const int64_t* line_g0;
  const int32_t* line_len;
  // the 32-cell, 128-byte aligned chunks of the padded grid that hold a
  // tissue-line cell (each once; vectors are allocated to a multiple of 32)
  int32_t n_chunks;
  const int32_t* chunk;
  // label | LAB_UNIFORM when all six neighbours carry the cell's own label
  // (and, with a smoothed boundary, psi is 1 at the cell and all six),
  // | LAB_PIN at the pinned voxel
  const uint8_t* label_u;
  // smoothed-boundary domain function per padded cell (0 off the rows), or
  // null for the sharp boundary
  const float* psi;
  // this handle's conductance tables (harmonic-mean face conductance / h^2,
  // HP_MAX_MATERIALS x HP_MAX_MATERIALS, FP32 for the iteration, FP64 for
  // the true residual): per handle, so that handles with different
  // conductivities can live side by side on one device
  const float* T32;
  const double* T64;
};

constexpr int LAB_UNIFORM = 0x80;
constexpr int LAB_PIN = 0x40;
constexpr int LAB_MASK = 0x3F;  // the material label (< HP_MAX_MATERIALS)
static_assert(HP_MAX_MATERIALS <= LAB_MASK + 1, "material labels must fit under the flag bits");

// Smoothed-boundary factor of a face: the harmonic mean of the two cells'
// domain function, 0 when both are 0 (build_torso_grid.py:350-375).
__device__ __forceinline__ float psi_face(float pa, float pb) {
  const float s = pa + pb;
  return s < 1e-30f ? 0.0f : __fdiv_rn(2.0f * pa * pb, s);
}
__host__ __device__ inline double psi_face64(double pa, double pb) {
  const double s = pa + pb;
  return s < 1e-30 ? 0.0 : (2.0 * pa * pb) / s;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

// Block-reduces NV values into part[blockIdx] -- slot q is a sum, or a max
// where bit q of max_mask is set (identity -inf) -- then returns true in the
// one block that arrived last, after which `tot` holds the grid totals in
// every thread of that block.
template <int NV>
__device__ bool block_reduce_last(double (&v)[NV], uint32_t max_mask, double* part,
                                  unsigned int* ticket, double (&tot)[NV]) {
  __shared__ double sh[TB / 32][NV];
  __shared__ bool am_last;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    const bool mx = (max_mask >> q) & 1u;
    double w = mx ? (double)warp_max((float)v[q]) : warp_sum(v[q]);
    if (lane == 0) sh[wid][q] = w;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      const bool mx = (max_mask >> q) & 1u;
      double s = sh[0][q];
      for (int w = 1; w < TB / 32; ++w) s = mx ? fmax(s, sh[w][q]) : s + sh[w][q];
      part[(int64_t)blockIdx.x * NPART + q] = s;
    }
    __threadfence();
    const unsigned int t = atomicAdd(ticket, 1u);
    am_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!am_last) return false;
  __threadfence();
  // the last block sums all partials in block order (deterministic)
#pragma unroll
  for (int q = 0; q < NV; ++q) v[q] = ((max_mask >> q) & 1u) ? -INFINITY : 0.0;
  for (int blk = threadIdx.x; blk < (int)gridDim.x; blk += TB) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      const double pv = ((volatile double*)part)[(int64_t)blk * NPART + q];
      v[q] = ((max_mask >> q) & 1u) ? fmax(v[q], pv) : v[q] + pv;
    }
  }
  // fixed-order tree over the block
  __shared__ double sh2[TB][NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) sh2[threadIdx.x][q] = v[q];
  __syncthreads();
  for (int s = TB / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
#pragma unroll
      for (int q = 0; q < NV; ++q)
        sh2[threadIdx.x][q] = ((max_mask >> q) & 1u)
                                  ? fmax(sh2[threadIdx.x][q], sh2[threadIdx.x + s][q])
                                  : sh2[threadIdx.x][q] + sh2[threadIdx.x + s][q];
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < NV; ++q) tot[q] = sh2[0][q];
  if (threadIdx.x == 0) *ticket = 0u;
  return true;
}

__device__ __forceinline__ bool is_row(const TorsoArgs& a, int64_t g) {
  return a.label[g] != 0 && g != a.pin;
}

// The PCG vector kernels walk tissue lines, one warp per line (lanes over
// consecutive k, coalesced rows), loading a batch of LB chunks of 32 cells
// before any arithmetic so every thread has several independent loads in
// flight.  Air lines are never touched; inside a line the vectors are zero
// on air cells and at the pinned voxel (r, p, x start at 0 and only row
// cells are ever written non-zero; invd is 0 there), so no labels are read.
template <int LB, class Load, class Apply>
__device__ __forceinline__ void for_line_batches(const TorsoArgs& a, Load&& load, Apply&& apply) {
  const int lane = threadIdx.x & 31;
  const int n_warps = gridDim.x * (TB / 32);
  for (int L = blockIdx.x * (TB / 32) + (threadIdx.x >> 5); L < a.n_lines; L += n_warps) {
    const int64_t g0 = a.line_g0[L];
    const int len = a.line_len[L];
    for (int k0 = lane; k0 < len; k0 += 32 * LB) {
#pragma unroll
      for (int u = 0; u < LB; ++u)
        if (k0 + 32 * u < len) load(u, g0 + k0 + 32 * u);
#pragma unroll
      for (int u = 0; u < LB; ++u)
        if (k0 + 32 * u < len) apply(u, g0 + k0 + 32 * u);
    }
  }
}

// The same over the chunk list: a warp takes U whole 32-cell chunks at a
// time, all loads issued before any arithmetic, every access a full
// 128-byte row segment.  Cells of a chunk outside every tissue line (air,
// the ends of the neighbouring rows) carry zeros in every vector and invd,
// so the updates leave them zero and they add nothing to the sums.
template <int U, class Load, class Apply>
__device__ __forceinline__ void for_chunk_batches(const TorsoArgs& a, Load&& load, Apply&& apply) {
  const int lane = threadIdx.x & 31;
  const int n_warps = gridDim.x * (TB / 32);
  const int w = blockIdx.x * (TB / 32) + (threadIdx.x >> 5);
  for (int c0 = w * U; c0 < a.n_chunks; c0 += n_warps * U) {
    int64_t g[U];
#pragma unroll
    for (int u = 0; u < U; ++u)
      g[u] = c0 + u < a.n_chunks ? (int64_t)a.chunk[c0 + u] * 32 + lane : -1;
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (g[u] >= 0) load(u, g[u]);
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (g[u] >= 0) apply(u, g[u]);
  }
}

// Iteration part 1a: pending x update and p <- M^-1 r + beta p, in place
// (every thread reads and writes only its own cells), over the chunk list
// (measured on the full torso: 28.7 us against 31.5 us over the tissue
// lines; the r update, with its FP64 sums, keeps the line batches of 8,
// which measured 24.2 us against 31.3 us over chunks).
__global__ void __launch_bounds__(TB, HP_PU_MINB) pcg_p_update(TorsoArgs a) {
  if (a.iscal[IS_DONE]) return;
  const double alpha_prev = a.scal[SC_ALPHA_PREV];
  const float betaf = (float)a.scal[SC_BETA];
  const float* __restrict__ invd = a.invd;
  const float* __restrict__ r = a.r;
  float* __restrict__ p = a.p0;
  double* __restrict__ x = a.x;
  constexpr int LB = 4;
  float pv[LB], zv[LB];
  if (alpha_prev != 0.0) {
    double xv[LB];
    for_chunk_batches<LB>(
        a, [&](int u, int64_t g) { pv[u] = p[g]; zv[u] = invd[g] * r[g]; xv[u] = x[g]; },
        [&](int u, int64_t g) {
          x[g] = xv[u] + alpha_prev * (double)pv[u];
          p[g] = zv[u] + betaf * pv[u];
        });
  } else {
    for_chunk_batches<LB>(
        a, [&](int u, int64_t g) { pv[u] = p[g]; zv[u] = invd[g] * r[g]; },
        [&](int u, int64_t g) { p[g] = zv[u] + betaf * pv[u]; });
  }
}

// Iteration part 1b: Ap = A p as a sum of face fluxes t (p_g - p_n) (exact
// for equal neighbours, so a smooth p keeps its small A p instead of a
// difference of two large sums), partial p.Ap; the last block forms alpha
// and clears the pending x update (part 1a applied it).  One warp per
// tissue line; all thirteen loads of a cell are issued before the sums
// (32-bit neighbour offsets keep the addressing to one base per array).
// The conductance table sits in shared memory (its reads diverge across a
// warp at material boundaries).  Measured and dropped on B200 (full torso,
// 5.8 M rows): a shared-memory 2.5-D blocked variant (8 x 32 columns
// marching 16 planes in i, 53-56 us against 37 us here: latency-bound at one
// plane in flight per block), two cells per thread (76 registers, 52 us) and
// a summed-difference path for uniform cells (40 us).
// Line SpMV core shared by the PCG and flexible-CG passes: Ap = A p over the
// tissue lines (Ap = 0 on air and at the pin), calling cell(g, p_g, Ap_g)
// for every cell; T is the conductance table in shared memory.
//
// Each lane takes two neighbouring cells of its line: the run is widened to
// start on an even cell (one air cell before the first tissue cell, and at
// most one after the last), so p, Ap and the labels of the pair move as one
// 8-byte / 2-byte access at the cell and at its four i / j neighbours (the
// padded plane and row strides are even), and the +-k neighbours come from
// the adjacent lanes by shuffles (lanes 0 and 31 load theirs).  Neighbour
// labels are read only where a cell's six neighbours do not all share its
// label.  Per-cell arithmetic is the same sum of face fluxes in the same
// face order as before.
template <bool PSI, class Cell>
__device__ __forceinline__ void spmv_lines(const TorsoArgs& a, const float* T, Cell&& cell) {
  const uint8_t* __restrict__ lab = a.label_u;
  const float* __restrict__ p = a.p0;
  float* __restrict__ Ap = a.Ap;
  const float* __restrict__ psi = a.psi;
  const int sj = a.pk, si = a.pj * a.pk;   // even; the padded plane fits in 32 bits
  const int lane = threadIdx.x & 31;
  const int n_warps = gridDim.x * (TB / 32);
  constexpr int M = LAB_MASK;
  for (int L = blockIdx.x * (TB / 32) + (threadIdx.x >> 5); L < a.n_lines; L += n_warps) {
    const int64_t g0 = a.line_g0[L];
    const int64_t ga = g0 & ~(int64_t)1;                  // even start
    const int npairs = (int)((g0 + a.line_len[L] - ga + 1) >> 1);
    for (int q0 = 0; q0 < npairs; q0 += 32) {
      const int q = q0 + lane;
      const bool on = q < npairs;
      const int64_t c = ga + 2 * (int64_t)q;            // first cell of the pair
      float2 pc = make_float2(0.0f, 0.0f), pip = pc, pim = pc, pjp = pc, pjm = pc;
      uchar2 lc = make_uchar2(0, 0);
      if (on) {
        pc = *(const float2*)(p + c);
        pip = *(const float2*)(p + c + si);
        pim = *(const float2*)(p + c - si);
        pjp = *(const float2*)(p + c + sj);
        pjm = *(const float2*)(p + c - sj);
        lc = *(const uchar2*)(lab + c);
      }
      // -k of the first cell = second cell of the lane below; +k of the
      // second cell = first cell of the lane above
      float km = __shfl_up_sync(0xffffffffu, pc.y, 1);
      float kp = __shfl_down_sync(0xffffffffu, pc.x, 1);
      if (on && lane == 0) km = p[c - 1];
      if (on && lane == 31) kp = p[c + 2];
      if (!on) continue;
      const float pv[2] = {pc.x, pc.y};
      const float pn0[2][6] = {{pip.x, pim.x, pjp.x, pjm.x, pc.y, km},
                               {pip.y, pim.y, pjp.y, pjm.y, kp, pc.x}};
      const int lf[2] = {lc.x, lc.y};
      float ap2[2];
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int l = lf[e] & M;
        // face conductances: one table entry inside a material region
        float tf[6];
        if (lf[e] & LAB_UNIFORM) {
          const float t = T[l * (HP_MAX_MATERIALS + 1)];
#pragma unroll
          for (int f = 0; f < 6; ++f) tf[f] = t;
        } else {
          const uint8_t* __restrict__ le = lab + c + e;
          const int off[6] = {si, -si, sj, -sj, 1, -1};
#pragma unroll
          for (int f = 0; f < 6; ++f) tf[f] = T[l * HP_MAX_MATERIALS + (le[off[f]] & M)];
          if constexpr (PSI) {
            const float* __restrict__ pe = psi + c + e;
            const float pself = pe[0];
#pragma unroll
            for (int f = 0; f < 6; ++f) tf[f] *= psi_face(pself, pe[off[f]]);
          }
        }
        float ap = 0.0f;
#pragma unroll
        for (int f = 0; f < 6; ++f) ap += tf[f] * (pv[e] - pn0[e][f]);
        if (l == 0 || (lf[e] & LAB_PIN)) ap = 0.0f;
        ap2[e] = ap;
      }
      *(float2*)(Ap + c) = make_float2(ap2[0], ap2[1]);
      cell(c, pv[0], ap2[0]);
      cell(c + 1, pv[1], ap2[1]);
    }
  }
}

// The same with one cell per lane, for a padded row of odd length (the
// pair accesses need even strides).
template <bool PSI, class Cell>
__device__ __forceinline__ void spmv_lines_single(const TorsoArgs& a, const float* T, Cell&& cell) {
  const uint8_t* __restrict__ lab = a.label_u;
  const float* __restrict__ p = a.p0;
  float* __restrict__ Ap = a.Ap;
  const float* __restrict__ psi = a.psi;
  const int sj = a.pk, si = a.pj * a.pk;   // the padded plane fits in 32 bits
  const int lane = threadIdx.x & 31;
  const int n_warps = gridDim.x * (TB / 32);
  for (int L = blockIdx.x * (TB / 32) + (threadIdx.x >> 5); L < a.n_lines; L += n_warps) {
    const int64_t g0 = a.line_g0[L];
    const int len = a.line_len[L];
    for (int k = lane; k < len; k += 32) {
      const int64_t g = g0 + k;
      const uint8_t* __restrict__ lc = lab + g;
      const float* __restrict__ pc = p + g;
      const int off[6] = {si, -si, sj, -sj, 1, -1};
      const int lf = lc[0];
      const int l = lf & LAB_MASK;
      const float pg = pc[0];
      float pn[6];
#pragma unroll
      for (int f = 0; f < 6; ++f) pn[f] = pc[off[f]];
      // inside a material region every face has the same conductance: one
      // table entry, and the neighbours' labels are read only at boundaries
      float tf[6];
      if (lf & LAB_UNIFORM) {
        const float t = T[l * (HP_MAX_MATERIALS + 1)];
#pragma unroll
        for (int f = 0; f < 6; ++f) tf[f] = t;
      } else {
#pragma unroll
        for (int f = 0; f < 6; ++f) tf[f] = T[l * HP_MAX_MATERIALS + (lc[off[f]] & LAB_MASK)];
        if constexpr (PSI) {
          const float pself = psi[g];
#pragma unroll
          for (int f = 0; f < 6; ++f) tf[f] *= psi_face(pself, psi[g + off[f]]);
        }
      }
      float ap = 0.0f;
#pragma unroll
      for (int f = 0; f < 6; ++f) ap += tf[f] * (pg - pn[f]);
      if (l == 0 || (lf & LAB_PIN)) ap = 0.0f;
      Ap[g] = ap;
      cell(g, pg, ap);
    }
  }
}

template <bool PAIRS, bool PSI>
__global__ void __launch_bounds__(TB, HP_AP_MINB) pcg_ap(TorsoArgs a) {
  __shared__ float T[HP_MAX_MATERIALS * HP_MAX_MATERIALS];
  if (a.iscal[IS_DONE]) return;
  for (int q = threadIdx.x; q < HP_MAX_MATERIALS * HP_MAX_MATERIALS; q += TB) T[q] = a.T32[q];
  __syncthreads();
  double acc[1] = {0.0};
  auto cell = [&](int64_t, float pg, float ap) { acc[0] += (double)pg * (double)ap; };
  if constexpr (PAIRS) spmv_lines<PSI>(a, T, cell);
  else spmv_lines_single<PSI>(a, T, cell);
  double tot[1];
  if (block_reduce_last<1>(acc, 0u, a.part, a.ticket, tot) && threadIdx.x == 0) {
    const double pAp = tot[0];
    a.scal[SC_PAP] = pAp;
    a.scal[SC_ALPHA_PREV] = 0.0;   // every block of part 1a applied the pending x update
    if (!(fabs(pAp) >= 1e-30) || !isfinite(pAp)) {   // breakdown, as the reference's |pAp| < 1e-30
      a.iscal[IS_BREAKDOWN] = isfinite(pAp) ? 1 : 0;
      a.iscal[IS_NONFINITE] = isfinite(pAp) ? 0 : 1;
      a.iscal[IS_DONE] = 1;
      a.scal[SC_ALPHA] = 0.0;
    } else {
      a.scal[SC_ALPHA] = a.scal[SC_RZ] / pAp;
    }
  }
}

// Iteration part 2: r -= alpha Ap, z = M^-1 r, partial r.z, z.z, r.r, max|z|;
// the last block forms beta and tests the stopping rule.
// P99 (the reference's 'p99' metric, compute_bspm.py:195-219): stop when the
// 0.99 quantile of |z| over the rows, linearly interpolated between order
// statistics as torch.quantile does, is below tol.  With N rows, position
// pos = 0.99 (N - 1), lo = floor(pos), and c rows at or above tol (their
// order statistics start at N - c), the quantile is below tol when lo + 1 <
// N - c, not below when lo >= N - c, and otherwise (lo = N - c - 1) equals
// m_lt + (pos - lo) (m_ge - m_lt) with m_lt the largest |z| below tol and
// m_ge the smallest at or above it: three reductions decide it exactly.
// The reported statistic is that value in the last case and otherwise
// m_lt (an upper bound of the quantile, below tol) or m_ge (a lower bound,
// not below tol).
template <bool P99>
__global__ void __launch_bounds__(TB, HP_K2_MINB) pcg_k2(TorsoArgs a) {
  if (a.iscal[IS_DONE]) return;
  const double alpha = a.scal[SC_ALPHA];
  const float alphaf = (float)alpha;
  const float tolf = (float)a.scal[SC_TOL];
  const float* __restrict__ invd = a.invd;
  const float* __restrict__ Ap = a.Ap;
  float* __restrict__ rv = a.r;
  // sums r.z, z.z, r.r and max |z|; P99: r.z, count |z| >= tol, max of |z|
  // below tol, max of -|z| at or above tol
  double acc[4] = {0.0, 0.0, P99 ? 0.0 : 0.0, P99 ? -INFINITY : 0.0};
  constexpr int LB = 8;
  float rb[LB], ib[LB];
  for_line_batches<LB>(
      a, [&](int u, int64_t g) { rb[u] = rv[g] - alphaf * Ap[g]; ib[u] = invd[g]; },
      [&](int u, int64_t g) {
        const float r = rb[u];
        rv[g] = r;
        const float z = ib[u] * r;
        acc[0] += (double)r * z;
        if constexpr (P99) {
          const float az = fabsf(z);
          if (az >= tolf) {
            acc[1] += 1.0;
            acc[3] = fmax(acc[3], -(double)az);
          } else {
            acc[2] = fmax(acc[2], (double)az);
          }
        } else {
          acc[1] += (double)z * z;
          acc[2] += (double)r * r;
          acc[3] = fmax(acc[3], (double)fabsf(z));
        }
      });
  double tot[4];
  if (block_reduce_last<4>(acc, P99 ? 12u : 8u, a.part, a.ticket, tot) && threadIdx.x == 0) {
    const double rz_new = tot[0];
    a.scal[SC_BETA] = rz_new / a.scal[SC_RZ];
    a.scal[SC_RZ] = rz_new;
    a.scal[SC_ALPHA_PREV] = alpha;
    const int it = ++a.iscal[IS_ITER];
    const int rule = a.iscal[IS_RULE];
    double stat;
    bool below;
    if constexpr (P99) {
      const double N = (double)a.n_rows, c = tot[1], m_lt = tot[2], m_ge = -tot[3];
      const double pos = 0.99 * (N - 1.0), lo = floor(pos);
      const double first_ge = N - c;
      if (lo + 1.0 < first_ge) {
        stat = m_lt;
        below = true;
      } else if (lo >= first_ge) {
        stat = m_ge;
        below = false;
      } else {
        stat = m_lt + (pos - lo) * (m_ge - m_lt);
        below = stat < a.scal[SC_TOL];
      }
    } else {
      a.scal[SC_ZZ] = tot[1];
      a.scal[SC_RR] = tot[2];
      a.scal[SC_ZMAX] = tot[3];
      if (rule == HP_STOP_RMS) stat = sqrt(tot[1] / (double)a.n_rows);
      else if (rule == HP_STOP_LINF) stat = tot[3];
      else stat = sqrt(tot[2] / fmax(a.scal[SC_BB], 1e-300));  // recursive estimate
      // REL: stop the recursion a little below tol; the true residual decides
      const double lim = rule == HP_STOP_REL ? 0.5 * a.scal[SC_TOL] : a.scal[SC_TOL];
      below = stat < lim;
    }
    a.scal[SC_STAT] = stat;
    if (!isfinite(rz_new)) { a.iscal[IS_NONFINITE] = 1; a.iscal[IS_DONE] = 1; }
    else if (below || it >= a.iscal[IS_MAXIT]) a.iscal[IS_DONE] = 1;
  }
}

// x += alpha_prev * p (the pending update of the last iteration).
__global__ void __launch_bounds__(TB) pcg_finish_x(TorsoArgs a) {
  const double alpha = a.scal[SC_ALPHA_PREV];
  const float* __restrict__ p = a.p0;
  for (int64_t g = blockIdx.x * (int64_t)TB + threadIdx.x; g < a.ng;
       g += (int64_t)gridDim.x * TB)
    if (is_row(a, g)) a.x[g] += alpha * (double)p[g];
}

// FP64 true residual r = b - A x (written to r in FP32), and ||r||^2,
// ||b||^2, r.M^-1 r.  Resets the CG recursion (beta = 0, no pending x).
__global__ void __launch_bounds__(TB) true_residual(TorsoArgs a, int reset) {
  const int64_t SJ = a.pk, SI = (int64_t)a.pj * a.pk;
  double acc[3] = {0.0, 0.0, 0.0};
  for (int64_t g = blockIdx.x * (int64_t)TB + threadIdx.x; g < a.ng;
       g += (int64_t)gridDim.x * TB) {
    if (!is_row(a, g)) continue;
    const int l = a.label[g];
    const int64_t nb[6] = {g + SI, g - SI, g + SJ, g - SJ, g + 1, g - 1};
    const double xg = a.x[g];
    double ax = 0.0;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      double t = a.T64[l * HP_MAX_MATERIALS + a.label[nb[f]]];
      if (a.psi) t *= psi_face64(a.psi[g], a.psi[nb[f]]);
      ax += t * (xg - a.x[nb[f]]);   // x is 0 on air and at the pinned voxel
    }
    const double bb = (double)a.b[g];
    const double rr = bb - ax;
    const float rf = (float)rr;
    if (reset) a.r[g] = rf;
    acc[0] += rr * rr;
    acc[1] += bb * bb;
    acc[2] += (double)rf * ((double)a.invd[g] * rf);
  }
  double tot[3];
  if (block_reduce_last<3>(acc, 0u, a.part, a.ticket, tot) && threadIdx.x == 0) {
    a.scal[SC_TRUE_RR] = tot[0];
    a.scal[SC_BB] = tot[1];
    if (reset) {
      a.scal[SC_RZ] = tot[2];
      a.scal[SC_BETA] = 0.0;
      a.scal[SC_ALPHA_PREV] = 0.0;
      a.iscal[IS_DONE] = 0;
    }
  }
}

// ---------------------------------------------------------------- sources

struct SrcArgs {
  int32_t n_heart;
  const int32_t* nbr;      // n_heart x 6
  const int32_t* proj;     // n_heart (coarse row or -1)
  const float* vm;         // n_heart, mV
  float* iv;               // n_heart: (sigma_i/h^2) K Vm (V) on projected voxels
  double coeff;
  double* part;
  unsigned int* ticket;
  double* scal;
  int64_t* mean_count;     // [1] number of projected voxels
};

// iv_i = coeff * sum_n (V_n - V_i) with V = Vm * 1e-3 volts (compute_bspm.py:381-387)
__global__ void __launch_bounds__(TB) src_laplacian(SrcArgs s) {
  double acc[1] = {0.0};
  for (int64_t i = blockIdx.x * (int64_t)TB + threadIdx.x; i < s.n_heart;
       i += (int64_t)gridDim.x * TB) {
    if (s.proj[i] < 0) continue;
    // differences of the mV values first (exact for equal neighbours), then
    // one scaling by 1e-3 * sigma_i / h^2
    const float vi = s.vm[i];
    float lap = 0.0f;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      const int32_t n = s.nbr[i * 6 + f];
      if (n >= 0) lap += __fsub_rn(s.vm[n], vi);
    }
    const float iv = lap * (float)(s.coeff * 1e-3);
    s.iv[i] = iv;
    acc[0] += (double)iv;
  }
  double tot[1];
  if (block_reduce_last<1>(acc, 0u, s.part, s.ticket, tot) && threadIdx.x == 0)
    s.scal[SC_SRC_MEAN] = tot[0] / (double)fmax(1.0, (double)*s.mean_count);
}

// b[row] = (sum of iv over the heart voxels of row - count * mean) / n_expected,
// one thread per receiving row (rows listed in seg order, deterministic).
__global__ void __launch_bounds__(TB) src_scatter(const float* iv, const int32_t* seg_ptr,
                                                  const int32_t* seg_vox, const int64_t* seg_grid,
                                                  int32_t n_seg, const double* scal,
                                                  double inv_nexp, float* b, int64_t pin,
                                                  const float* psi) {
  const int q = blockIdx.x * TB + threadIdx.x;
  if (q >= n_seg) return;
  const float mean = (float)scal[SC_SRC_MEAN];
  float s = 0.0f;
  for (int t = seg_ptr[q]; t < seg_ptr[q + 1]; ++t) s += iv[seg_vox[t]] - mean;
  const int64_t g = seg_grid[q];
  float bg = (float)(s * inv_nexp);
  if (psi) bg *= psi[g];   // smoothed boundary: psi b (compute_bspm.py:413-414)
  b[g] = g == pin ? 0.0f : bg;
}

__global__ void gather_out(const double* x, const int64_t* grid_of_read, int32_t n, float* out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) out[q] = (float)(x[grid_of_read[q]] * 1e3);
}

__global__ void gather_rows(const double* x, const int64_t* grid_of_row, int64_t n, double* out) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q < n) out[q] = x[grid_of_row[q]];
}

__global__ void gather_rows_f(const float* b, const int64_t* grid_of_row, int64_t n, float* out) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q < n) out[q] = b[grid_of_row[q]];
}

// flexible-CG passes (defined with the FCG driver below)
template <bool PAIRS>
__global__ void __launch_bounds__(TB) fcg_spmv(TorsoArgs a);
__global__ void __launch_bounds__(TB) fcg_update(TorsoArgs a);
__global__ void __launch_bounds__(TB) fcg_beta(TorsoArgs a);
__global__ void __launch_bounds__(TB) fcg_p(TorsoArgs a, int first);

}  // namespace hp

using namespace hp;

// kernels that stride over the tissue lines, in the order of HpTorso::nblk_k
enum LineKernel : int { K_P_UPDATE = 0, K_AP, K_K2, K_FCG_SPMV, K_FCG_UPDATE, K_FCG_BETA, K_FCG_P,
                        N_LINE_KERNELS };

struct HpTorso {
  TorsoArgs a;
  SrcArgs s;
  int nblk;
  int nblk_k[N_LINE_KERNELS];  // line kernels: each one's resident grid
  bool pairs;                  // stencil on cell pairs (even padded row)
  void (*ap_fn)(TorsoArgs);
  void (*fspmv_fn)(TorsoArgs);
  int ni, nj, nk;
  int64_t n_rows;
  std::vector<void*> allocs;
  int32_t n_read;
  int64_t* grid_of_read;
  int64_t* grid_of_row;
  int32_t* seg_ptr;
  int32_t* seg_vox;
  int64_t* seg_grid;
  int32_t n_seg;
  double inv_nexp;
  float* vm_dev;
  float* out_dev;
  double* h_scal;   // pinned host mirrors
  int32_t* h_iscal;
  int parity;
  bool have_x;
  cudaGraphExec_t graph[2];
  cudaGraphExec_t fcg_graph[4];   // FCG chunk without the network / net every 1, 2, 4
  // serial number of the preconditioner handle the FCG graphs hold (not its
  // address: a destroyed handle's address can come back for a new one, whose
  // buffers the old graphs do not point to)
  uint64_t fcg_graph_pc;
  cudaStream_t fcg_graph_stream;
  int graph_chunk;
  cudaStream_t graph_stream;
};

template <typename T>
static hp_status tup(HpTorso* h, T** dst, const T* src, size_t n, cudaStream_t s) {
  hp_status st = dev_upload(dst, src, n, s);
  if (st == HP_OK && *dst) h->allocs.push_back((void*)*dst);
  return st;
}
template <typename T>
static hp_status tal(HpTorso* h, T** dst, size_t n) {
  hp_status st = dev_alloc(dst, n);
  if (st == HP_OK && *dst) h->allocs.push_back((void*)*dst);
  return st;
}

#define TT_TRY(x)                \
  do {                           \
    hp_status _s = (x);          \
    if (_s != HP_OK) {           \
      hp_torso_destroy(h);       \
      return _s;                 \
    }                            \
  } while (0)

extern "C" hp_status hp_torso_create(const HpTorsoDesc* d, HpTorso** out, void* stream) {
  HP_REQUIRE(d && out, "hp_torso_create: null argument");
  *out = nullptr;
  HP_REQUIRE(d->ni > 0 && d->nj > 0 && d->nk > 0 && d->label, "hp_torso_create: empty grid");
  HP_REQUIRE(d->n_materials >= 1 && d->n_materials <= HP_MAX_MATERIALS && d->sigma,
             "hp_torso_create: n_materials must be 1..%d", HP_MAX_MATERIALS);
  HP_REQUIRE(d->h_m > 0.0, "hp_torso_create: h_m must be positive");
  HP_REQUIRE(d->n_heart >= 0 && (d->n_heart == 0 || (d->heart_nbr && d->proj)),
             "hp_torso_create: missing heart arrays");
  HP_REQUIRE(d->n_read >= 0 && (d->n_read == 0 || d->read_rows), "hp_torso_create: missing read_rows");
  cudaStream_t s = (cudaStream_t)stream;
  const int ni = d->ni, nj = d->nj, nk = d->nk;
  const int PI = ni + 2, PJ = nj + 2, PK = nk + 2;
  const int64_t ng = (int64_t)PI * PJ * PK;
  // padded labels (and smoothed-boundary psi), row <-> grid maps (rows in
  // flat active order)
  std::vector<uint8_t> lab(ng, 0);
  std::vector<float> psi(d->psi ? ng : 0, 0.0f);
  std::vector<int64_t> grid_of_row;
  grid_of_row.reserve((size_t)ni * nj * nk);
  for (int i = 0; i < ni; ++i)
    for (int j = 0; j < nj; ++j)
      for (int k = 0; k < nk; ++k) {
        const uint8_t l = d->label[((int64_t)i * nj + j) * nk + k];
        if (l >= d->n_materials) {
          hp::set_error("hp_torso_create: label %d at (%d,%d,%d) >= n_materials", l, i, j, k);
          return HP_ERR_INVALID;
        }
        const int64_t g = ((int64_t)(i + 1) * PJ + (j + 1)) * PK + (k + 1);
        lab[g] = l;
        if (l != 0) grid_of_row.push_back(g);
        if (d->psi) {
          const float pv = d->psi[((int64_t)i * nj + j) * nk + k];
          if (!(pv >= 0.0f && pv <= 1.0f) || (pv > 0.0f) != (l != 0)) {
            hp::set_error("hp_torso_create: psi %g at (%d,%d,%d) must be in (0, 1] exactly where "
                          "the label is non-zero (label %d)", (double)pv, i, j, k, l);
            return HP_ERR_INVALID;
          }
          psi[g] = pv;
        }
      }
  const int64_t n_rows = (int64_t)grid_of_row.size();
  HP_REQUIRE(d->pin_row >= 0 && d->pin_row < n_rows, "hp_torso_create: pin_row out of range");
  for (int m = 0; m < d->n_read; ++m)
    HP_REQUIRE(d->read_rows[m] >= 0 && d->read_rows[m] < n_rows,
               "hp_torso_create: read_rows[%d] out of range", m);
  // conductance tables (harmonic mean / h^2; both-zero pairs -> 0)
  float T32[HP_MAX_MATERIALS * HP_MAX_MATERIALS] = {0};
  double T64[HP_MAX_MATERIALS * HP_MAX_MATERIALS] = {0};
  const double h2 = d->h_m * d->h_m;
  for (int u = 0; u < d->n_materials; ++u)
    for (int v = 0; v < d->n_materials; ++v) {
      const double su = d->sigma[u], sv = d->sigma[v];
      if (u == 0 || v == 0 || su + sv < 1e-30) continue;   // air never couples
      const double g = (2.0 * su * sv) / (su + sv) / h2;
      T64[u * HP_MAX_MATERIALS + v] = g;
      T32[u * HP_MAX_MATERIALS + v] = (float)g;
    }
  // Jacobi inverse diagonal (FP32 of the FP64 diagonal), 0 on the pin
  const int64_t SJ = PK, SI = (int64_t)PJ * PK;
  std::vector<float> invd(ng, 0.0f);
  const int64_t pin_g = grid_of_row[d->pin_row];
  for (int64_t r = 0; r < n_rows; ++r) {
    const int64_t g = grid_of_row[r];
    if (g == pin_g) continue;
    const int l = lab[g];
    const int64_t nb[6] = {g + SI, g - SI, g + SJ, g - SJ, g + 1, g - 1};
    double dg = 0.0;
    for (int f = 0; f < 6; ++f)
      dg += T64[l * HP_MAX_MATERIALS + lab[nb[f]]] *
            (d->psi ? psi_face64(psi[g], psi[nb[f]]) : 1.0);
    invd[g] = dg > 1e-30 ? (float)(1.0 / dg) : 1.0f;
  }
  HpTorso* h = new HpTorso();
  memset(&h->a, 0, sizeof(h->a));
  memset(&h->s, 0, sizeof(h->s));
  h->graph[0] = h->graph[1] = nullptr;
  h->graph_chunk = 0;
  h->graph_stream = nullptr;
  for (int k = 0; k < 4; ++k) h->fcg_graph[k] = nullptr;
  h->fcg_graph_pc = 0;
  h->fcg_graph_stream = nullptr;
  h->ni = ni; h->nj = nj; h->nk = nk;
  h->n_rows = n_rows;
  h->parity = 0;
  h->have_x = false;
  TorsoArgs& a = h->a;
  TT_TRY(tup(h, (float**)&a.T32, T32, HP_MAX_MATERIALS * HP_MAX_MATERIALS, s));
  TT_TRY(tup(h, (double**)&a.T64, T64, HP_MAX_MATERIALS * HP_MAX_MATERIALS, s));
  a.ng = ng; a.pj = PJ; a.pk = PK; a.pin = pin_g; a.n_rows = n_rows;
  // the vectors and invd extend to a multiple of 32 cells (whole chunks),
  // zero past the grid
  const int64_t ng32 = (ng + 31) / 32 * 32;
  invd.resize(ng32, 0.0f);
  TT_TRY(tup(h, (uint8_t**)&a.label, lab.data(), ng, s));
  TT_TRY(tup(h, (float**)&a.invd, invd.data(), ng32, s));
  a.psi = nullptr;
  if (d->psi) TT_TRY(tup(h, (float**)&a.psi, psi.data(), ng, s));
  TT_TRY(tal(h, &a.r, ng32));
  TT_TRY(tal(h, &a.p0, ng32));
  TT_TRY(tal(h, &a.p1, ng32));
  TT_TRY(tal(h, &a.Ap, ng32));
  TT_TRY(tal(h, &a.x, ng32));
  TT_TRY(tal(h, &a.b, ng32));
  HP_CUDA_TRY(cudaMemsetAsync(a.r, 0, ng32 * 4, s));
  HP_CUDA_TRY(cudaMemsetAsync(a.p0, 0, ng32 * 4, s));
  HP_CUDA_TRY(cudaMemsetAsync(a.p1, 0, ng32 * 4, s));
  HP_CUDA_TRY(cudaMemsetAsync(a.Ap, 0, ng32 * 4, s));
  HP_CUDA_TRY(cudaMemsetAsync(a.x, 0, ng32 * 8, s));
  HP_CUDA_TRY(cudaMemsetAsync(a.b, 0, ng32 * 4, s));
  int nsm = 148;
  {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  }
  h->nblk = nsm * 8;
  {
    // the line loops stride over the grid, so a grid larger than what is
    // resident would leave a tail wave: each kernel gets its resident grid
    int o = 0;
    // cell pairs need even padded strides (an even padded row)
    h->pairs = (PK % 2) == 0;
    // the smoothed-boundary face weights are a separate instantiation, so
    // the sharp operator carries no psi code
    h->ap_fn = a.psi ? (h->pairs ? pcg_ap<true, true> : pcg_ap<false, true>)
                     : (h->pairs ? pcg_ap<true, false> : pcg_ap<false, false>);
    h->fspmv_fn = h->pairs ? fcg_spmv<true> : fcg_spmv<false>;
    const void* fs[N_LINE_KERNELS] = {(const void*)pcg_p_update, (const void*)h->ap_fn,
                                      (const void*)pcg_k2<false>, (const void*)h->fspmv_fn,
                                      (const void*)fcg_update,   (const void*)fcg_beta,
                                      (const void*)fcg_p};
    for (int q = 0; q < N_LINE_KERNELS; ++q) {
      HP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, fs[q], TB, 0));
      h->nblk_k[q] = nsm * std::min(8, std::max(o, 1));
    }
  }
  TT_TRY(tal(h, &a.scal, N_SCAL));
  TT_TRY(tal(h, &a.iscal, N_ISCAL));
  TT_TRY(tal(h, &a.part, (size_t)h->nblk * NPART));
  TT_TRY(tal(h, &a.ticket, 1));
  HP_CUDA_TRY(cudaMemsetAsync(a.scal, 0, N_SCAL * 8, s));
  HP_CUDA_TRY(cudaMemsetAsync(a.iscal, 0, N_ISCAL * 4, s));
  HP_CUDA_TRY(cudaMemsetAsync(a.ticket, 0, 4, s));
  TT_TRY(tup(h, &h->grid_of_row, grid_of_row.data(), n_rows, s));
  {
    // tissue lines of the padded grid: first .. last tissue cell in k
    std::vector<int64_t> g0;
    std::vector<int32_t> len;
    for (int i = 1; i <= ni; ++i)
      for (int j = 1; j <= nj; ++j) {
        const int64_t base = ((int64_t)i * PJ + j) * PK;
        int k0 = -1, k1 = -1;
        for (int k = 1; k <= nk; ++k)
          if (lab[base + k] != 0) {
            if (k0 < 0) k0 = k;
            k1 = k;
          }
        if (k0 >= 0) {
          g0.push_back(base + k0);
          len.push_back(k1 - k0 + 1);
        }
      }
    a.n_lines = (int32_t)g0.size();
    // chunks: the 32-cell aligned blocks that a tissue line touches, each once
    std::vector<int32_t> chunks;
    for (size_t L = 0; L < g0.size(); ++L) {
      const int64_t c0 = g0[L] >> 5, c1 = (g0[L] + len[L] - 1) >> 5;
      for (int64_t c = c0; c <= c1; ++c)
        if (chunks.empty() || chunks.back() < (int32_t)c) chunks.push_back((int32_t)c);
    }
    a.n_chunks = (int32_t)chunks.size();
    std::vector<uint8_t> lab_u(lab);
    for (int64_t r = 0; r < n_rows; ++r) {
      const int64_t g = grid_of_row[r];
      const int64_t nb[6] = {g + SI, g - SI, g + SJ, g - SJ, g + 1, g - 1};
      bool uni = !d->psi || psi[g] == 1.0f;
      for (int f = 0; f < 6; ++f)
        uni = uni && lab[nb[f]] == lab[g] && (!d->psi || psi[nb[f]] == 1.0f);
      if (uni) lab_u[g] |= (uint8_t)LAB_UNIFORM;
    }
    lab_u[pin_g] |= (uint8_t)LAB_PIN;
    TT_TRY(tup(h, (uint8_t**)&a.label_u, lab_u.data(), lab_u.size(), s));

    TT_TRY(tup(h, (int64_t**)&a.line_g0, g0.data(), g0.size(), s));
    TT_TRY(tup(h, (int32_t**)&a.line_len, len.data(), len.size(), s));
    TT_TRY(tup(h, (int32_t**)&a.chunk, chunks.data(), chunks.size(), s));
    HP_CUDA_TRY(cudaStreamSynchronize(s));  // g0 / len / chunks are stack temporaries
  }
  // heart sources: segments of heart voxels per receiving row
  SrcArgs& sa = h->s;
  sa.n_heart = d->n_heart;
  sa.coeff = d->coeff;
  sa.part = a.part;
  sa.ticket = a.ticket;
  sa.scal = a.scal;
  h->inv_nexp = 1.0 / d->n_expected;
  std::vector<int32_t> order;
  int64_t n_valid = 0;
  for (int32_t i = 0; i < d->n_heart; ++i) {
    if (d->proj[i] >= n_rows) {
      hp::set_error("hp_torso_create: proj[%d]=%d out of range", i, d->proj[i]);
      hp_torso_destroy(h);
      return HP_ERR_INVALID;
    }
    for (int f = 0; f < 6; ++f) {
      const int32_t nbv = d->heart_nbr[(int64_t)i * 6 + f];
      if (nbv >= d->n_heart) {
        hp::set_error("hp_torso_create: heart_nbr out of range at %d", i);
        hp_torso_destroy(h);
        return HP_ERR_INVALID;
      }
    }
    if (d->proj[i] >= 0) { order.push_back(i); ++n_valid; }
  }
  std::stable_sort(order.begin(), order.end(),
                   [&](int32_t u, int32_t v) { return d->proj[u] < d->proj[v]; });
  std::vector<int32_t> seg_ptr(1, 0), seg_vox;
  std::vector<int64_t> seg_grid;
  for (size_t t = 0; t < order.size(); ++t) {
    if (t > 0 && d->proj[order[t]] != d->proj[order[t - 1]]) {
      seg_ptr.push_back((int32_t)t);
    }
    if (t == 0 || d->proj[order[t]] != d->proj[order[t - 1]])
      seg_grid.push_back(grid_of_row[d->proj[order[t]]]);
    seg_vox.push_back(order[t]);
  }
  seg_ptr.push_back((int32_t)order.size());
  if (order.empty()) seg_ptr.assign(1, 0);
  h->n_seg = (int32_t)seg_grid.size();
  TT_TRY(tup(h, &h->seg_ptr, seg_ptr.data(), seg_ptr.size(), s));
  TT_TRY(tup(h, &h->seg_vox, seg_vox.data(), seg_vox.size(), s));
  TT_TRY(tup(h, &h->seg_grid, seg_grid.data(), seg_grid.size(), s));
  TT_TRY(tup(h, (int32_t**)&sa.nbr, d->heart_nbr, (size_t)d->n_heart * 6, s));
  TT_TRY(tup(h, (int32_t**)&sa.proj, d->proj, d->n_heart, s));
  TT_TRY(tal(h, &h->vm_dev, d->n_heart));
  TT_TRY(tal(h, &sa.iv, d->n_heart));
  if (d->n_heart) HP_CUDA_TRY(cudaMemsetAsync(sa.iv, 0, d->n_heart * 4, s));
  TT_TRY(tup(h, &sa.mean_count, &n_valid, 1, s));
  sa.vm = h->vm_dev;
  // read-out rows
  h->n_read = d->n_read;
  std::vector<int64_t> gr(d->n_read);
  for (int m = 0; m < d->n_read; ++m) gr[m] = grid_of_row[d->read_rows[m]];
  TT_TRY(tup(h, &h->grid_of_read, gr.data(), gr.size(), s));
  TT_TRY(tal(h, &h->out_dev, d->n_read));
  HP_CUDA_TRY(cudaMallocHost((void**)&h->h_scal, N_SCAL * sizeof(double)));
  HP_CUDA_TRY(cudaMallocHost((void**)&h->h_iscal, N_ISCAL * sizeof(int32_t)));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  *out = h;
  return HP_OK;
}

extern "C" int64_t hp_torso_rows(const HpTorso* h) { return h ? h->n_rows : -1; }

static hp_status iter_launch(HpTorso* h, int n, bool p99, cudaStream_t s) {
  for (int q = 0; q < n; ++q) {
    pcg_p_update<<<h->nblk_k[K_P_UPDATE], TB, 0, s>>>(h->a);
    h->ap_fn<<<h->nblk_k[K_AP], TB, 0, s>>>(h->a);
    if (p99) pcg_k2<true><<<h->nblk_k[K_K2], TB, 0, s>>>(h->a);
    else pcg_k2<false><<<h->nblk_k[K_K2], TB, 0, s>>>(h->a);
  }
  HP_CUDA_TRY(cudaGetLastError());
  return HP_OK;
}

// CG iterations in chunks of `chunk` (one CUDA graph per stopping-rule
// kernel: graph[1] for the p99 rule), with the host reading the done flag
// once per chunk.  Kernels after convergence inside a chunk return
// immediately.
static hp_status run_iterations(HpTorso* h, int max_iter, bool p99, cudaStream_t s) {
  const int chunk = 8;
  const int gi = p99 ? 1 : 0;
  if (s == nullptr) {    // the legacy default stream cannot be captured
    for (int done_it = 0; done_it < max_iter + chunk; done_it += chunk) {
      hp_status st = iter_launch(h, chunk, p99, s);
      if (st != HP_OK) return st;
      HP_CUDA_TRY(cudaMemcpyAsync(h->h_iscal, h->a.iscal, N_ISCAL * 4, cudaMemcpyDeviceToHost, s));
      HP_CUDA_TRY(cudaStreamSynchronize(s));
      if (h->h_iscal[IS_DONE]) break;
    }
    return HP_OK;
  }
  if (h->graph_stream != s) {
    for (int k = 0; k < 2; ++k) {
      if (h->graph[k]) cudaGraphExecDestroy(h->graph[k]);
      h->graph[k] = nullptr;
    }
    h->graph_stream = s;
  }
  if (!h->graph[gi]) {
    cudaGraph_t g;
    HP_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    hp_status st = iter_launch(h, chunk, p99, s);
    cudaError_t ce = cudaStreamEndCapture(s, &g);
    if (st != HP_OK) return st;
    HP_CUDA_TRY(ce);
    HP_CUDA_TRY(cudaGraphInstantiate(&h->graph[gi], g, 0));
    cudaGraphDestroy(g);
    h->graph_chunk = chunk;
  }
  for (int done_it = 0; done_it < max_iter + chunk; done_it += chunk) {
    HP_CUDA_TRY(cudaGraphLaunch(h->graph[gi], s));
    HP_CUDA_TRY(cudaMemcpyAsync(h->h_iscal, h->a.iscal, N_ISCAL * 4, cudaMemcpyDeviceToHost, s));
    HP_CUDA_TRY(cudaStreamSynchronize(s));
    if (h->h_iscal[IS_DONE]) break;
  }
  return HP_OK;
}

namespace hp {

// b <- per-frame source (compute_bspm.py:381-419)
static hp_status build_rhs(HpTorso* h, const float* vm, int vm_on_device, cudaStream_t s) {
  TorsoArgs& a = h->a;
  SrcArgs& sa = h->s;
  if (sa.n_heart > 0) {
    HP_REQUIRE(vm, "torso solve: vm is null");
    HP_CUDA_TRY(cudaMemcpyAsync(h->vm_dev, vm, (size_t)sa.n_heart * 4,
                                vm_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
  }
  HP_CUDA_TRY(cudaMemsetAsync(a.b, 0, a.ng * 4, s));
  if (sa.n_heart > 0) {
    src_laplacian<<<h->nblk, TB, 0, s>>>(sa);
    if (h->n_seg > 0)
      src_scatter<<<(h->n_seg + TB - 1) / TB, TB, 0, s>>>(sa.iv, h->seg_ptr, h->seg_vox,
                                                           h->seg_grid, h->n_seg, a.scal,
                                                           h->inv_nexp, a.b, a.pin, a.psi);
  }
  HP_CUDA_TRY(cudaGetLastError());
  return HP_OK;
}

static hp_status read_scalars(HpTorso* h, cudaStream_t s) {
  HP_CUDA_TRY(cudaMemcpyAsync(h->h_scal, h->a.scal, N_SCAL * 8, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaMemcpyAsync(h->h_iscal, h->a.iscal, N_ISCAL * 4, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  return HP_OK;
}

// Jacobi-PCG from the current x on the current b.  *result receives the
// outcome (HP_OK, NOT_CONVERGED, STAGNATED, NONFINITE).
static hp_status pcg_solve(HpTorso* h, double tol, int rule, int max_iter, HpSolveStats* stats,
                           hp_status* result_out, cudaStream_t s) {
  TorsoArgs& a = h->a;
  double tol_dev = rule == HP_STOP_REL ? tol : tol * 1e-3;   // mV -> V for the mV rules
  HP_CUDA_TRY(cudaMemcpyAsync(a.scal + SC_TOL, &tol_dev, 8, cudaMemcpyHostToDevice, s));
  int32_t is_init[N_ISCAL] = {0, 0, rule, max_iter, 0, 0};
  HP_CUDA_TRY(cudaMemcpyAsync(a.iscal, is_init, sizeof(is_init), cudaMemcpyHostToDevice, s));
  // r = b - A x0 (warm start; x = 0 for the first frame), beta = 0
  true_residual<<<h->nblk, TB, 0, s>>>(a, 1);
  HP_CUDA_TRY(cudaGetLastError());
  int restarts = 0;
  int total_it = 0;
  hp_status result = HP_OK;
  double rel = 0.0;
  for (;;) {
    HP_CUDA_TRY(cudaMemcpyAsync(h->h_scal, a.scal, N_SCAL * 8, cudaMemcpyDeviceToHost, s));
    HP_CUDA_TRY(cudaStreamSynchronize(s));
    const double bb = h->h_scal[SC_BB];
    rel = bb > 0.0 ? sqrt(h->h_scal[SC_TRUE_RR] / bb) : 0.0;
    if (bb == 0.0 && rule == HP_STOP_REL) {   // zero source: the pinned solution is 0
      HP_CUDA_TRY(cudaMemsetAsync(a.x, 0, a.ng * 8, s));
      rel = 0.0;
      break;
    }
    if (rule == HP_STOP_REL && rel <= tol) break;
    if (total_it >= max_iter) { result = HP_ERR_NOT_CONVERGED; break; }
    int32_t is_run[N_ISCAL] = {0, 0, rule, max_iter - total_it, 0, 0};
    HP_CUDA_TRY(cudaMemcpyAsync(a.iscal, is_run, sizeof(is_run), cudaMemcpyHostToDevice, s));
    hp_status st = run_iterations(h, max_iter - total_it, rule == HP_STOP_P99, s);
    if (st != HP_OK) return st;
    st = read_scalars(h, s);
    if (st != HP_OK) return st;
    const int its = h->h_iscal[IS_ITER];
    total_it += its;
    if (its > 0) {
      pcg_finish_x<<<h->nblk, TB, 0, s>>>(a);
      HP_CUDA_TRY(cudaGetLastError());
    }
    if (h->h_iscal[IS_NONFINITE]) { result = HP_ERR_NONFINITE; break; }
    if (rule != HP_STOP_REL) {
      // reference mV rules: the recursive statistic decides
      true_residual<<<h->nblk, TB, 0, s>>>(a, 0);
      HP_CUDA_TRY(cudaMemcpyAsync(h->h_scal, a.scal, N_SCAL * 8, cudaMemcpyDeviceToHost, s));
      HP_CUDA_TRY(cudaStreamSynchronize(s));
      rel = h->h_scal[SC_BB] > 0 ? sqrt(h->h_scal[SC_TRUE_RR] / h->h_scal[SC_BB]) : 0.0;
      if (!(h->h_scal[SC_STAT] < tol_dev)) result = HP_ERR_NOT_CONVERGED;
      if (h->h_iscal[IS_BREAKDOWN]) result = HP_OK;   // reference: break, return x
      break;
    }
    // relative rule: the true residual decides; replace r and restart if needed
    true_residual<<<h->nblk, TB, 0, s>>>(a, 1);
    HP_CUDA_TRY(cudaGetLastError());
    ++restarts;
    if (restarts > 50) { result = HP_ERR_STAGNATED; break; }
  }
  if (rule == HP_STOP_REL && restarts > 0) --restarts;   // the final check is not a restart
  if (stats) {
    stats->iterations = total_it;
    stats->status = result;
    stats->rel_residual = rel;
    stats->stat = h->h_scal[SC_STAT];
    stats->restarts = restarts;
  }
  *result_out = result;
  return HP_OK;
}

static hp_status readout(HpTorso* h, float* out, int out_on_device, cudaStream_t s) {
  if (h->n_read > 0 && out) {
    gather_out<<<(h->n_read + 255) / 256, 256, 0, s>>>(h->a.x, h->grid_of_read, h->n_read,
                                                        out_on_device ? out : h->out_dev);
    if (!out_on_device)
      HP_CUDA_TRY(cudaMemcpyAsync(out, h->out_dev, h->n_read * 4, cudaMemcpyDeviceToHost, s));
  }
  HP_CUDA_TRY(cudaGetLastError());
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  return HP_OK;
}

static hp_status finish(hp_status result, const char* what) {
  if (result == HP_ERR_NOT_CONVERGED || result == HP_ERR_STAGNATED) return HP_OK;  // in stats
  if (result != HP_OK) {
    hp::set_error("%s: non-finite values in the solve", what);
    return result;
  }
  return HP_OK;
}

}  // namespace hp

extern "C" hp_status hp_torso_solve_frame(HpTorso* h, const float* vm, int32_t vm_on_device,
                                          float* out, int32_t out_on_device, double tol,
                                          int32_t rule, int32_t max_iter, HpSolveStats* stats,
                                          void* stream) {
  HP_REQUIRE(h, "hp_torso_solve_frame: null handle");
  HP_REQUIRE(rule >= 0 && rule <= 3, "hp_torso_solve_frame: unknown rule %d", rule);
  HP_REQUIRE(max_iter >= 1, "hp_torso_solve_frame: max_iter must be >= 1");
  HP_REQUIRE(tol > 0.0, "hp_torso_solve_frame: tol must be positive");
  cudaStream_t s = (cudaStream_t)stream;
  hp_status st = build_rhs(h, vm, vm_on_device, s);
  if (st != HP_OK) return st;
  hp_status result = HP_OK;
  st = pcg_solve(h, tol, rule, max_iter, stats, &result, s);
  if (st != HP_OK) return st;
  st = readout(h, out, out_on_device, s);
  if (st != HP_OK) return st;
  h->have_x = true;
  return finish(result, "hp_torso_solve_frame");
}

extern "C" hp_status hp_torso_arrays(HpTorso* h, HpTorsoArrays* o) {
  HP_REQUIRE(h && o, "hp_torso_arrays: null argument");
  o->ni = h->ni; o->nj = h->nj; o->nk = h->nk;
  o->n_cells = h->a.ng;
  o->pin_cell = h->a.pin;
  o->label = h->a.label;
  o->invd = h->a.invd;
  o->r = h->a.r;
  o->x = h->a.x;
  o->b = h->a.b;
  return HP_OK;
}

// ------------------------------------------------------------ flexible CG

namespace hp {
namespace pc {
hp_status precond_apply(HpPrecond* h, const uint8_t* label, const float* invd, const float* r,
                        float* z, int use_net, cudaStream_t s);
uint64_t precond_serial(const HpPrecond* h);
}

// q = A p (p in p0), partial p.q and p.r; last block: alpha = p.r / p.q.
// The flexible-CG passes walk the tissue lines like the PCG ones (the
// preconditioner output z is zero on air and at the pin as well).
template <bool PAIRS>
__global__ void __launch_bounds__(TB) fcg_spmv(TorsoArgs a) {
  __shared__ float T[HP_MAX_MATERIALS * HP_MAX_MATERIALS];
  if (a.iscal[IS_DONE]) return;
  for (int q = threadIdx.x; q < HP_MAX_MATERIALS * HP_MAX_MATERIALS; q += TB) T[q] = a.T32[q];
  __syncthreads();
  const float* __restrict__ rv = a.r;
  double acc[2] = {0.0, 0.0};
  auto cell = [&](int64_t g, float pv, float q) {
    acc[0] += (double)pv * q;
    acc[1] += (double)pv * rv[g];
  };
  if constexpr (PAIRS) spmv_lines<false>(a, T, cell);
  else spmv_lines_single<false>(a, T, cell);
  double tot[2];
  if (block_reduce_last<2>(acc, 0u, a.part, a.ticket, tot) && threadIdx.x == 0) {
    a.scal[SC_PAP] = tot[0];
    if (!(fabs(tot[0]) >= 1e-30) || !isfinite(tot[0])) {
      a.iscal[IS_BREAKDOWN] = isfinite(tot[0]) ? 1 : 0;
      a.iscal[IS_NONFINITE] = isfinite(tot[0]) ? 0 : 1;
      a.iscal[IS_DONE] = 1;
      a.scal[SC_ALPHA] = 0.0;
    } else {
      a.scal[SC_ALPHA] = tot[1] / tot[0];
    }
  }
}

// x += alpha p, r -= alpha q, partial r.r; last block: recursive stat, done test
__global__ void __launch_bounds__(TB) fcg_update(TorsoArgs a) {
  if (a.iscal[IS_DONE]) return;
  const double alpha = a.scal[SC_ALPHA];
  const float af = (float)alpha;
  const float* __restrict__ p = a.p0;
  const float* __restrict__ Ap = a.Ap;
  float* __restrict__ rv = a.r;
  double* __restrict__ x = a.x;
  double acc[1] = {0.0};
  constexpr int LB = 4;
  float pb[LB], rb[LB];
  double xb[LB];
  for_line_batches<LB>(
      a,
      [&](int u, int64_t g) {
        pb[u] = p[g];
        xb[u] = x[g];
        rb[u] = rv[g] - af * Ap[g];
      },
      [&](int u, int64_t g) {
        x[g] = xb[u] + alpha * (double)pb[u];
        rv[g] = rb[u];
        acc[0] += (double)rb[u] * rb[u];
      });
  double tot[1];
  if (block_reduce_last<1>(acc, 0u, a.part, a.ticket, tot) && threadIdx.x == 0) {
    a.scal[SC_RR] = tot[0];
    const double stat = sqrt(tot[0] / fmax(a.scal[SC_BB], 1e-300));
    a.scal[SC_STAT] = stat;
    const int it = ++a.iscal[IS_ITER];
    // stagnation: less than 3 % progress over the last 5 iterations
    const int nh = ++a.iscal[IS_NH];
    a.scal[SC_HIST0 + (nh - 1) % 8] = stat;
    const bool stagnant =
        a.iscal[IS_STAG_ON] && nh > 6 && stat > 0.97 * a.scal[SC_HIST0 + (nh - 6) % 8];
    if (!isfinite(tot[0])) { a.iscal[IS_NONFINITE] = 1; a.iscal[IS_DONE] = 1; }
    else if (stat < 0.5 * a.scal[SC_TOL] || it >= a.iscal[IS_MAXIT]) a.iscal[IS_DONE] = 1;
    else if (stagnant) { a.iscal[IS_STAGNANT] = 1; a.iscal[IS_DONE] = 1; }
  }
}

// partial z.q (z in p1); last block: beta = -z.q / p.q
__global__ void __launch_bounds__(TB) fcg_beta(TorsoArgs a) {
  const float* __restrict__ z = a.p1;
  const float* __restrict__ Ap = a.Ap;
  double acc[1] = {0.0};
  constexpr int LB = 8;
  float zb[LB], qb[LB];
  for_line_batches<LB>(
      a, [&](int u, int64_t g) { zb[u] = z[g]; qb[u] = Ap[g]; },
      [&](int u, int64_t) { acc[0] += (double)zb[u] * qb[u]; });
  double tot[1];
  if (block_reduce_last<1>(acc, 0u, a.part, a.ticket, tot) && threadIdx.x == 0)
    a.scal[SC_BETA] = -tot[0] / a.scal[SC_PAP];
}

// p = z + beta p
__global__ void __launch_bounds__(TB) fcg_p(TorsoArgs a, int first) {
  const float beta = first ? 0.0f : (float)a.scal[SC_BETA];
  const float* __restrict__ z = a.p1;
  float* __restrict__ p = a.p0;
  constexpr int LB = 8;
  float zb[LB], pb[LB];
  for_line_batches<LB>(
      a, [&](int u, int64_t g) { zb[u] = z[g]; pb[u] = p[g]; },
      [&](int u, int64_t g) { p[g] = zb[u] + beta * pb[u]; });
}

__global__ void error_kernel(TorsoArgs a, const double* __restrict__ xstar, float* __restrict__ e) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < a.ng;
       g += (int64_t)gridDim.x * blockDim.x)
    e[g] = is_row(a, g) ? (float)(xstar[g] - a.x[g]) : 0.0f;
}

constexpr int FCG_CHUNK = 4;

// The FCG iteration body (A p, x / r update and stopping tests, z = M(r),
// beta, p) for FCG_CHUNK iterations, captured once per network period,
// stream and preconditioner handle.  use_net = k > 0 applies the network
// term on every k-th iteration of the chunk (k divides FCG_CHUNK) and the
// Jacobi + coarse terms alone on the others: flexible CG admits a
// preconditioner that changes from one iteration to the next.
static hp_status fcg_graph(HpTorso* h, HpPrecond* p, int use_net, cudaStream_t s) {
  const int q = use_net == 0 ? 0 : (use_net == 1 ? 1 : (use_net == 2 ? 2 : 3));
  const uint64_t serial = pc::precond_serial(p);
  if (h->fcg_graph[q] && h->fcg_graph_stream == s && h->fcg_graph_pc == serial)
    return HP_OK;
  if (h->fcg_graph_stream != s || h->fcg_graph_pc != serial) {
    for (int k = 0; k < 4; ++k)
      if (h->fcg_graph[k]) { cudaGraphExecDestroy(h->fcg_graph[k]); h->fcg_graph[k] = nullptr; }
  }
  TorsoArgs& a = h->a;
  cudaGraph_t g;
  HP_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  hp_status st = HP_OK;
  for (int it = 0; it < FCG_CHUNK && st == HP_OK; ++it) {
    h->fspmv_fn<<<h->nblk_k[K_FCG_SPMV], TB, 0, s>>>(a);
    fcg_update<<<h->nblk_k[K_FCG_UPDATE], TB, 0, s>>>(a);
    st = pc::precond_apply(p, a.label, a.invd, a.r, a.p1, use_net > 0 && it % use_net == 0, s);
    if (st != HP_OK) break;
    fcg_beta<<<h->nblk_k[K_FCG_BETA], TB, 0, s>>>(a);
    fcg_p<<<h->nblk_k[K_FCG_P], TB, 0, s>>>(a, 0);
  }
  cudaError_t ce = cudaStreamEndCapture(s, &g);
  if (st != HP_OK) return st;
  HP_CUDA_TRY(ce);
  HP_CUDA_TRY(cudaGraphInstantiate(&h->fcg_graph[q], g, 0));
  cudaGraphDestroy(g);
  h->fcg_graph_stream = s;
  h->fcg_graph_pc = serial;
  return HP_OK;
}

// One flexible-CG run with M (use_net selects the network term) from the
// current x; returns with *fallback set when it did not converge within
// fallback_iter iterations, stagnated or broke down.
static hp_status fcg_run(HpTorso* h, HpPrecond* p, double tol, int fallback_iter, int use_net,
                         int* it_out, int* restarts_out, double* rel_out, bool* fallback,
                         cudaStream_t s) {
  TorsoArgs& a = h->a;
  *fallback = false;
  HP_CUDA_TRY(cudaMemcpyAsync(a.scal + SC_TOL, &tol, 8, cudaMemcpyHostToDevice, s));
  // the stagnation test guards the runs with the network; the method
  // without it runs until convergence or the iteration budget
  int32_t is_init[N_ISCAL] = {0, 0, HP_STOP_REL, fallback_iter, 0, 0};
  is_init[IS_STAG_ON] = use_net ? 1 : 0;
  HP_CUDA_TRY(cudaMemcpyAsync(a.iscal, is_init, sizeof(is_init), cudaMemcpyHostToDevice, s));
  true_residual<<<h->nblk, TB, 0, s>>>(a, 1);
  HP_CUDA_TRY(cudaGetLastError());
  hp_status st = read_scalars(h, s);
  if (st != HP_OK) return st;
  const double bb = h->h_scal[SC_BB];
  double rel = bb > 0.0 ? sqrt(h->h_scal[SC_TRUE_RR] / bb) : 0.0;
  int it = 0;
  if (bb == 0.0) {
    HP_CUDA_TRY(cudaMemsetAsync(a.x, 0, a.ng * 8, s));
    *rel_out = 0.0;
    *it_out = 0;
    return HP_OK;
  }
  // chunks of FCG_CHUNK iterations replayed from a CUDA graph; kernels of a
  // chunk after the device-side done flag return at once (the
  // preconditioner's then only writes its own scratch and z)
  // z = M(r0), p = z (this first application also sets up anything the
  // preconditioner initialises lazily, before the capture)
  st = pc::precond_apply(p, a.label, a.invd, a.r, a.p1, use_net, s);
  if (st != HP_OK) return st;
  fcg_p<<<h->nblk_k[K_FCG_P], TB, 0, s>>>(a, 1);
  st = fcg_graph(h, p, use_net, s);
  if (st != HP_OK) return st;
  bool restart = false;
  while (rel > tol) {
    if (restart) {
      st = pc::precond_apply(p, a.label, a.invd, a.r, a.p1, use_net, s);
      if (st != HP_OK) return st;
      fcg_p<<<h->nblk_k[K_FCG_P], TB, 0, s>>>(a, 1);
      restart = false;
    }
    HP_CUDA_TRY(cudaGraphLaunch(h->fcg_graph[use_net == 0 ? 0 : (use_net == 1 ? 1 : (use_net == 2 ? 2 : 3))], s));
    st = read_scalars(h, s);
    if (st != HP_OK) return st;
    it = h->h_iscal[IS_ITER];
    if (h->h_iscal[IS_NONFINITE] || h->h_iscal[IS_BREAKDOWN] || h->h_iscal[IS_STAGNANT]) {
      *fallback = true;
      break;
    }
    if (h->h_iscal[IS_DONE]) {
      if (h->h_scal[SC_STAT] >= 0.5 * tol) { *fallback = true; break; }   // iteration budget
      // recursive residual below tol / 2: the FP64 true residual decides
      true_residual<<<h->nblk, TB, 0, s>>>(a, 1);
      st = read_scalars(h, s);
      if (st != HP_OK) return st;
      rel = sqrt(h->h_scal[SC_TRUE_RR] / h->h_scal[SC_BB]);
      if (rel <= tol) break;
      ++*restarts_out;
      int32_t is_re[N_ISCAL] = {0, it, HP_STOP_REL, fallback_iter, 0, 0};
      is_re[IS_STAG_ON] = use_net ? 1 : 0;
      HP_CUDA_TRY(cudaMemcpyAsync(a.iscal, is_re, sizeof(is_re), cudaMemcpyHostToDevice, s));
      restart = true;
    }
  }
  *it_out = it;
  *rel_out = rel;
  return HP_OK;
}

// Flexible CG with the learned preconditioner.  Safeguards, in order: when
// the run with the network fails (no convergence within fallback_iter,
// stagnation or breakdown), FCG restarts from the current iterate without
// the network (the two-level method, restarts += 100; no stagnation test,
// up to max(fallback_iter, 1000) iterations); when that fails too, plain
// Jacobi-PCG finishes the frame (restarts += 1000).
static hp_status fcg_solve(HpTorso* h, HpPrecond* p, double tol, int max_iter, int fallback_iter,
                           int use_net, HpSolveStats* stats, hp_status* result_out, cudaStream_t s) {
  int it_total = 0, restarts = 0;
  double rel = 0.0;
  bool fallback = false;
  hp_status result = HP_OK;
  // the run with the network (use_net = its period) for at most
  // fallback_iter iterations, then without it (the two-level method, which
  // converges on its own: up to 1000 iterations, or fallback_iter if more)
  for (int net = use_net; net >= 0; net = net > 0 ? 0 : -1) {
    int it = 0;
    const int cap = net > 0 ? fallback_iter : std::max(fallback_iter, 1000);
    const int budget = std::max(1, std::min(cap, max_iter - it_total));
    hp_status st = fcg_run(h, p, tol, budget, net, &it, &restarts, &rel, &fallback, s);
    if (st != HP_OK) return st;
    it_total += it;
    if (!fallback) break;
    if (net > 0) restarts += 100;
  }
  if (fallback) {
    HpSolveStats st2;
    hp_status r2 = HP_OK;
    hp_status st = pcg_solve(h, tol, HP_STOP_REL, std::max(1, max_iter - it_total), &st2, &r2, s);
    if (st != HP_OK) return st;
    it_total += st2.iterations;
    rel = st2.rel_residual;
    result = r2;
    restarts += 1000;
  }
  if (stats) {
    stats->iterations = it_total;
    stats->status = result;
    stats->rel_residual = rel;
    stats->stat = rel;
    stats->restarts = restarts;
  }
  *result_out = result;
  return HP_OK;
}

}  // namespace hp

extern "C" hp_status hp_torso_solve_frame_fcg(HpTorso* h, HpPrecond* p, const float* vm,
                                              int32_t vm_on_device, float* out,
                                              int32_t out_on_device, double tol, int32_t max_iter,
                                              int32_t fallback_iter, int32_t use_net,
                                              HpSolveStats* stats, void* stream) {
  HP_REQUIRE(h, "hp_torso_solve_frame_fcg: null torso handle");
  HP_REQUIRE(!h->a.psi, "hp_torso_solve_frame_fcg: the flexible-CG preconditioners are built for "
                        "the sharp-boundary operator; a smoothed-boundary (psi) handle solves "
                        "with hp_torso_solve_frame");
  HP_REQUIRE(p, "hp_torso_solve_frame_fcg: null preconditioner");
  HP_REQUIRE(max_iter >= 1 && fallback_iter >= 1, "hp_torso_solve_frame_fcg: bad iteration limits");
  HP_REQUIRE(use_net == 0 || use_net == 1 || use_net == 2 || use_net == 4,
             "hp_torso_solve_frame_fcg: use_net must be 0, 1, 2 or 4");
  HP_REQUIRE(tol > 0.0, "hp_torso_solve_frame_fcg: tol must be positive");
  cudaStream_t s = (cudaStream_t)stream;
  hp_status st = build_rhs(h, vm, vm_on_device, s);
  if (st != HP_OK) return st;
  hp_status result = HP_OK;
  st = fcg_solve(h, p, tol, max_iter, fallback_iter, use_net, stats, &result, s);
  if (st != HP_OK) return st;
  st = readout(h, out, out_on_device, s);
  if (st != HP_OK) return st;
  h->have_x = true;
  return finish(result, "hp_torso_solve_frame_fcg");
}

namespace hp {
// n more iterations of the current CG recursion (no restart, no stopping
// test), then the pending x update applied so that x is the n-th iterate.
static hp_status pcg_continue(HpTorso* h, int n, cudaStream_t s) {
  TorsoArgs& a = h->a;
  const double never = 0.0;     // relative rule with tolerance 0: runs all n
  HP_CUDA_TRY(cudaMemcpyAsync(a.scal + SC_TOL, &never, 8, cudaMemcpyHostToDevice, s));
  int32_t is_run[N_ISCAL] = {0, 0, HP_STOP_REL, n, 0, 0};
  HP_CUDA_TRY(cudaMemcpyAsync(a.iscal, is_run, sizeof(is_run), cudaMemcpyHostToDevice, s));
  hp_status st = run_iterations(h, n, false, s);
  if (st != HP_OK) return st;
  pcg_finish_x<<<h->nblk, TB, 0, s>>>(a);
  HP_CUDA_TRY(cudaGetLastError());
  const double zero = 0.0;      // the update is applied: nothing pending
  HP_CUDA_TRY(cudaMemcpyAsync(a.scal + SC_ALPHA_PREV, &zero, 8, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));   // the host scalars above are stack temporaries
  return HP_OK;
}
}  // namespace hp

extern "C" hp_status hp_torso_train_precond(HpTorso* h, HpPrecond* p, const float* vm_frames,
                                            int64_t frame_stride, int32_t n_frames,
                                            const int32_t* ks, int32_t n_ks, int32_t repeats,
                                            float lr, double tol_exact, float* loss_hist,
                                            void* stream) {
  HP_REQUIRE(h && !h->a.psi, "hp_torso_train_precond: the preconditioners are built for the "
                            "sharp-boundary operator (this handle has psi)");
  HP_REQUIRE(h && p && vm_frames && ks && n_frames >= 1 && n_ks >= 1 && repeats >= 1,
             "hp_torso_train_precond: bad arguments");
  for (int q = 0; q < n_ks; ++q)
    HP_REQUIRE(ks[q] >= 0 && (q == 0 || ks[q] >= ks[q - 1]),
               "hp_torso_train_precond: ks must be non-negative and ascending");
  cudaStream_t s = (cudaStream_t)stream;
  TorsoArgs& a = h->a;
  double *xstar = nullptr, *x0 = nullptr;
  float* e = nullptr;
  HP_CUDA_TRY(cudaMalloc((void**)&xstar, a.ng * 8));
  HP_CUDA_TRY(cudaMalloc((void**)&x0, a.ng * 8));
  HP_CUDA_TRY(cudaMalloc((void**)&e, a.ng * 4));
  hp_status ret = HP_OK;
  int64_t q = 0;
  for (int f = 0; f < n_frames && ret == HP_OK; ++f) {
    ret = build_rhs(h, vm_frames + (int64_t)f * frame_stride, 1, s);
    if (ret != HP_OK) break;
    if (cudaMemcpyAsync(x0, a.x, a.ng * 8, cudaMemcpyDeviceToDevice, s) != cudaSuccess) { ret = HP_ERR_CUDA; break; }
    hp_status res = HP_OK;
    ret = pcg_solve(h, tol_exact, HP_STOP_REL, 20000, nullptr, &res, s);
    if (ret != HP_OK) break;
    if (cudaMemcpyAsync(xstar, a.x, a.ng * 8, cudaMemcpyDeviceToDevice, s) != cudaSuccess) { ret = HP_ERR_CUDA; break; }
    // one plain-PCG trajectory from the warm start; pairs at iterations ks
    // (ascending): r_k (the recursion's residual) and e_k = x* - x_k
    if (cudaMemcpyAsync(a.x, x0, a.ng * 8, cudaMemcpyDeviceToDevice, s) != cudaSuccess) { ret = HP_ERR_CUDA; break; }
    true_residual<<<h->nblk, TB, 0, s>>>(a, 1);     // r = b - A x0, fresh recursion
    int done = 0;
    for (int kq = 0; kq < n_ks && ret == HP_OK; ++kq) {
      if (ks[kq] > done) {
        ret = pcg_continue(h, ks[kq] - done, s);
        if (ret != HP_OK) break;
        done = ks[kq];
      }
      error_kernel<<<h->nblk, TB, 0, s>>>(a, xstar, e);
      for (int rp = 0; rp < repeats && ret == HP_OK; ++rp) {
        float loss = 0.0f;
        ret = hp_precond_train_step(p, a.label, a.invd, a.r, e, lr, &loss, s);
        if (loss_hist) loss_hist[q] = loss;
        ++q;
      }
    }
    if (ret == HP_OK && cudaMemcpyAsync(a.x, xstar, a.ng * 8, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
      ret = HP_ERR_CUDA;
  }
  cudaStreamSynchronize(s);
  cudaFree(xstar);
  cudaFree(x0);
  cudaFree(e);
  return ret;
}

extern "C" hp_status hp_torso_copy_solution(HpTorso* h, double* x_rows, void* stream) {
  HP_REQUIRE(h && x_rows, "hp_torso_copy_solution: null argument");
  cudaStream_t s = (cudaStream_t)stream;
  double* tmp = nullptr;
  HP_CUDA_TRY(cudaMalloc((void**)&tmp, h->n_rows * 8));
  gather_rows<<<(unsigned)((h->n_rows + 255) / 256), 256, 0, s>>>(h->a.x, h->grid_of_row,
                                                                  h->n_rows, tmp);
  HP_CUDA_TRY(cudaMemcpyAsync(x_rows, tmp, h->n_rows * 8, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  HP_CUDA_TRY(cudaFree(tmp));
  return HP_OK;
}

extern "C" hp_status hp_torso_copy_rhs(HpTorso* h, float* b_rows, void* stream) {
  HP_REQUIRE(h && b_rows, "hp_torso_copy_rhs: null argument");
  cudaStream_t s = (cudaStream_t)stream;
  float* tmp = nullptr;
  HP_CUDA_TRY(cudaMalloc((void**)&tmp, h->n_rows * 4));
  gather_rows_f<<<(unsigned)((h->n_rows + 255) / 256), 256, 0, s>>>(h->a.b, h->grid_of_row,
                                                                    h->n_rows, tmp);
  HP_CUDA_TRY(cudaMemcpyAsync(b_rows, tmp, h->n_rows * 4, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  HP_CUDA_TRY(cudaFree(tmp));
  return HP_OK;
}

extern "C" hp_status hp_torso_reset(HpTorso* h) {
  HP_REQUIRE(h, "hp_torso_reset: null handle");
  HP_CUDA_TRY(cudaMemset(h->a.x, 0, h->a.ng * 8));
  h->have_x = false;
  return HP_OK;
}

extern "C" hp_status hp_torso_destroy(HpTorso* h) {
  if (!h) return HP_OK;
  for (int q = 0; q < 2; ++q)
    if (h->graph[q]) cudaGraphExecDestroy(h->graph[q]);
  for (int q = 0; q < 4; ++q)
    if (h->fcg_graph[q]) cudaGraphExecDestroy(h->fcg_graph[q]);
  for (void* p : h->allocs) cudaFree(p);
  if (h->h_scal) cudaFreeHost(h->h_scal);
  if (h->h_iscal) cudaFreeHost(h->h_iscal);
  delete h;
  return HP_OK;
}
