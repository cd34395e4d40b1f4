// Fused monodomain time step for sm_100a.
//
// One launch advances every myocardial voxel and every Purkinje node by one
// step of the reference's Lie splitting at theta = 0
// (simulation/functions/purkinje_myocardium_pipeline.py:1347-1420,
//  anisotropic_simulation/functions/purkinje_myocardium_anisotropic_solver.py:1746-1820):
//
//   V*_i     = V_i + dt/Cm (-Iion(V_i) Cm + Istim_i)          (ionic half)
//   V_{i+1}  = clamp(V*_i + dt/Cm * L V*_i, -150, 80)           (diffusion half)
//
// The kernel is skewed by half a step so that a single pass per voxel is
// enough: launch i reads W_i = V*_i of the voxel and its 18 neighbours,
// forms V_{i+1} (recording threshold crossings and snapshots on it), then
// immediately runs the TTP06 update of step i+1 on V_{i+1} and stores
// W_{i+1}.  A prologue launch (mode 1) produces W_0 from the resting state.
// W is double-buffered (neighbours need the old value); V_{i+1} is kept in
// Vpost for the crossing test of the next step and for snapshots.
//
// Data layout in HBM (see include/hrdaya_b200.h): voxels of the mask in
// bricks of BI x BJ x BK with k fastest, only bricks that touch the mask are
// stored; every per-voxel field is a separate SoA array over slots, so each
// warp's loads and stores are contiguous 128-byte lines.  The stencil reads
// W (and, for the 19-point operator, the face weights and off-diagonal
// tensor components) of the brick plus a one-voxel halo into shared memory.
#include "hp_common.cuh"
#include "ttp06.cuh"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#include <algorithm>
#include <vector>

namespace hp {

struct MonoArgs {
  int32_t n_bricks, n_pk;
  int64_t n_slots;
  const uint32_t* tag;
  const float* wface;  // 3 x n_slots
  const float* doff;   // 3 x n_slots
  float iso_coef;
  const int32_t* nbr;  // n_bricks x 27
  const uint8_t* brick_variant;
  float* state;        // 18 x n_slots
  float* Vs0;                       // W double buffer (slots)
  float* Vs1;
  float* Vpost;
  // Purkinje
  const int32_t* pk_ptr;
  const int32_t* pk_idx;
  const float* pk_coef;
  const uint8_t* pk_stim;
  const uint8_t* pk_variant;
  float* pk_state;     // 18 x n_pk
  float* pk_Vs0;
  float* pk_Vs1;
  float* pk_Vpost;
  // junctions, myocardial side
  const int32_t* pmj_row;
  const int32_t* pmj_ptr;
  const int32_t* pmj_pk;
  const float* pmj_coef;
  // time stepping
  double dt_d;
  float dt, Cm, dt_over_Cm;
  const float* site_amp;     // n_variants x HP_MAX_SITES, uA/mm^2
  const uint8_t* site_on;    // n_variants x site_stride pulse bitmasks
  int64_t site_stride;       // n_steps + 1
  const float* var_gks;
  const float* var_gkr;
  // outputs
  float* vm_snap;
  const int32_t* node_of_slot;
  int64_t vm_every, n_myo;
  float* surf_frames;
  const int32_t* surf_of_slot;
  int64_t n_surf;
  float* pk_frames;
  int64_t frame_every;
  float act_thr, deact_thr;
  int32_t max_events;
  float* act_t;
  uint8_t* act_n;
  float* deact_t;
  uint8_t* deact_n;
  const int64_t* d_step;
  // pipelined kernel: halo copy table of the brick shape
  int32_t n_halo;
  const uint32_t* halo_tab;
  // split step: tissue slots in increasing order, the Purkinje threads start
  // at n_active_pad (n_active rounded up to a warp); slot >> bv_shift = brick
  int32_t n_active, n_active_pad, bv_shift;
  const int32_t* active_slot;
  // theta-scheme: the CG solution x ([slots | Purkinje]) of the step
  const float* cn_x;
};

// TTP06 phenotype table (ttp06_phenotype_constants.py:54-61), index = pheno-1.
__device__ __forceinline__ CellParams pheno_params(int ph, float gks_s, float gkr_s) {
  CellParams p;
  p.g_Kr = 0.153f * gkr_s;
  if (ph == 1) {         // endo
    p.g_Ks = 0.392f * gks_s; p.g_to = 0.073f; p.endo_s = 1;
  } else if (ph == 2) {  // mid
    p.g_Ks = 0.098f * gks_s; p.g_to = 0.294f; p.endo_s = 1;
  } else {               // epi
    p.g_Ks = 0.392f * gks_s; p.g_to = 0.294f; p.endo_s = 0;
  }
  return p;
}

// Stimulus current of a cell of variant var at step istep: the sum of the
// amplitudes of its sites that fire then (each variant has its own sites).
__device__ __forceinline__ float stim_current(const MonoArgs& a, uint32_t bits, int64_t istep,
                                              int var) {
  uint32_t on = bits & (uint32_t)a.site_on[var * a.site_stride + istep];
  float I = 0.0f;
  while (on) {
    int s = __ffs(on) - 1;
    I += a.site_amp[var * HP_MAX_SITES + s];
    on &= on - 1;
  }
  return I;
}

// One threshold crossing between snapshots (t0, v0) -> (t1, v1), linear
// interpolation as activation_maps.py:63-89 (float32, frac clipped to [0,1]).
__device__ __forceinline__ void record_event(float* tbl, uint8_t* cnt, int64_t slot,
                                             int64_t n_slots, int max_events, float thr,
                                             float v0, float v1, float t0, float t1) {
  float den = v1 - v0;
  if (den == 0.0f) den = 1e-9f;
  float frac = __fdiv_rn(thr - v0, den);
  frac = fminf(fmaxf(frac, 0.0f), 1.0f);
  const float tc = __fadd_rn(t0, __fmul_rn(frac, __fsub_rn(t1, t0)));
  const int n = cnt[slot];
  if (n < max_events) tbl[(int64_t)n * n_slots + slot] = tc;
  if (n < 255) cnt[slot] = (uint8_t)(n + 1);
}

template <int BI, int BJ, int BK>
struct TileGeom {
  static constexpr int TI = BI + 2, TJ = BJ + 2, TK = BK + 2;
  static constexpr int N = TI * TJ * TK;
  static constexpr int SI = TJ * TK, SJ = TK;
  static constexpr int BV = BI * BJ * BK;
};

// Loads local region [I0,I1) x [J0,J1) x [K0,K1) (coordinates relative to the
// brick, -1 and B* address the halo) of a slot array into a shared tile.
template <int BI, int BJ, int BK, int I0, int I1, int J0, int J1, int K0, int K1>
__device__ __forceinline__ void load_region(float* __restrict__ tile,
                                            const float* __restrict__ src,
                                            const int* nb27, int tid) {
  using G = TileGeom<BI, BJ, BK>;
  constexpr int NI = I1 - I0, NJ = J1 - J0, NK = K1 - K0, NT = NI * NJ * NK;
#pragma unroll 4
  for (int e = tid; e < NT; e += G::BV) {
    const int ek = e % NK;
    const int t = e / NK;
    const int ej = t % NJ;
    const int ei = t / NJ;
    const int li = ei + I0, lj = ej + J0, lk = ek + K0;
    const int di = li < 0 ? -1 : (li >= BI ? 1 : 0);
    const int dj = lj < 0 ? -1 : (lj >= BJ ? 1 : 0);
    const int dk = lk < 0 ? -1 : (lk >= BK ? 1 : 0);
    const int nb = nb27[(di + 1) * 9 + (dj + 1) * 3 + (dk + 1)];
    float v = 0.0f;
    if (nb >= 0) {
      const int gi = li - di * BI, gj = lj - dj * BJ, gk = lk - dk * BK;
      v = __ldg(src + (int64_t)nb * G::BV + (gi * BJ + gj) * BK + gk);
    }
    tile[(li + 1) * G::SI + (lj + 1) * G::SJ + (lk + 1)] = v;
  }
}

// Purkinje nodes: thread per node over the CSR adjacency (cable edges and
// junction edges to myocardial slots), same skewed step as the voxels.
// Diffusion half: V_{i+1} of node p from W_i, stored in pk_Vpost (and the
// animation frame of step i).
// Row sum of Purkinje node p: sum_q coef_q (W_j - W_p) over its cable and
// junction edges (Purkinje potentials in Wpk, myocardial ones in Wmyo).
// DIAG: the diagonal of the row instead (every difference reads -1).
template <bool DIAG = false>
__device__ __forceinline__ float purkinje_acc(const MonoArgs& a, int p,
                                              const float* __restrict__ Wpk,
                                              const float* __restrict__ Wmyo) {
  const float Vc = DIAG ? 0.0f : Wpk[p];
  float acc = 0.0f;
  for (int q = a.pk_ptr[p]; q < a.pk_ptr[p + 1]; ++q) {
    if constexpr (DIAG) {
      acc += a.pk_coef[q] * -1.0f;
    } else {
      const int j = a.pk_idx[q];
      const float Vj = j >= 0 ? Wpk[j] : Wmyo[-(int64_t)j - 1];
      acc += a.pk_coef[q] * (Vj - Vc);
    }
  }
  return acc;
}

__device__ __forceinline__ float purkinje_diffuse(const MonoArgs& a, int p, int64_t step) {
  const bool odd = step & 1;
  const float* __restrict__ Win = odd ? a.pk_Vs1 : a.pk_Vs0;
  const float* __restrict__ Wmyo = odd ? a.Vs1 : a.Vs0;
  const float Vc = Win[p];
  const float acc = purkinje_acc(a, p, Win, Wmyo);
  const float Vn = fminf(fmaxf(Vc + acc, -150.0f), 80.0f);
  a.pk_Vpost[p] = Vn;
  if (a.frame_every > 0 && step % a.frame_every == 0)
    a.pk_frames[(step / a.frame_every) * (int64_t)a.n_pk + p] = Vn;
  return Vn;
}

// Ionic half of step istep of node p on V = Vn with its state c; stores the
// state and W.
__device__ __forceinline__ void purkinje_ionic_state(const MonoArgs& a, int p, float Vn,
                                                     CellState& c, int64_t istep,
                                                     float* __restrict__ Wout) {
  const int var = a.pk_variant ? a.pk_variant[p] : 0;
  const CellParams cp = pheno_params(1, a.var_gks[var], a.var_gkr[var]);  // Purkinje -> endo
  const float Iion = ttp06_step(Vn, c, a.dt, cp);
#pragma unroll
  for (int v = 0; v < N_STATE; ++v) a.pk_state[(int64_t)v * a.n_pk + p] = c.v[v];
  const float Is = stim_current(a, a.pk_stim[p], istep, var);
  Wout[p] = Vn + a.dt_over_Cm * (-(Iion * a.Cm) + Is);
}

__device__ __forceinline__ void purkinje_ionic(const MonoArgs& a, int p, float Vn, int64_t istep,
                                               float* __restrict__ Wout) {
  CellState c;
#pragma unroll
  for (int v = 0; v < N_STATE; ++v) c.v[v] = a.pk_state[(int64_t)v * a.n_pk + p];
  purkinje_ionic_state(a, p, Vn, c, istep, Wout);
}

__device__ __forceinline__ void purkinje_part(const MonoArgs& a, int p, int64_t step, int mode) {
  const bool odd = step & 1;
  if (mode == 0) {
    const float Vn = purkinje_diffuse(a, p, step);
    purkinje_ionic(a, p, Vn, step + 1, odd ? a.pk_Vs0 : a.pk_Vs1);
  } else {
    purkinje_ionic(a, p, a.pk_Vpost[p], 0, a.pk_Vs0);
  }
}

// Operator sum of one voxel from its operands, in one fixed order of
// explicitly rounded operations, so every kernel that feeds it (shared-memory
// tiles, registers) gets bit-identical results.  nv(q) is the value of
// neighbour q: the faces +i, -i, +j, -j, +k, -k (q = 0..5), then the twelve
// edge neighbours in diagonal-bit order (q = 6..17); wf(f) the weight of face
// f; tc(e) and tn(e) the off-diagonal tensor component of edge term e at the
// voxel and at its edge neighbour.  Face and diagonal bits of the tag gate
// every term.  The co-signed edge pairs (+,+)/(-,-) carry +avg, the
// counter-signed ones -avg (bit e has the minus sign when e & 2).
// DIAG: every difference reads -1, so the sum is the operator's diagonal.
template <bool ANISO, bool DIAG, class NV, class WF, class TC, class TN>
__device__ __forceinline__ float stencil_sum(float iso_coef, uint32_t tag, float Vc, NV&& nv,
                                             WF&& wf, TC&& tc, TN&& tn) {
#define HP_DV(x) (DIAG ? -1.0f : __fsub_rn((x), Vc))
  const uint32_t fb = tag >> HP_TAG_FACE_SHIFT;
  float acc = 0.0f;
  if constexpr (!ANISO) {
    float s = 0.0f;
#pragma unroll
    for (int f = 0; f < 6; ++f)
      if (fb & (1u << f)) s = __fadd_rn(s, HP_DV(nv(f)));
    acc = __fmul_rn(iso_coef, s);
  } else {
#pragma unroll
    for (int f = 0; f < 6; ++f)
      if (fb & (1u << f)) acc = __fmaf_rn(wf(f), HP_DV(nv(f)), acc);
    const uint32_t db = tag >> HP_TAG_DIAG_SHIFT;
#pragma unroll
    for (int e = 0; e < 12; ++e)
      if (db & (1u << e))
        acc = __fmaf_rn(__fmul_rn((e & 2) ? -0.25f : 0.25f, __fadd_rn(tc(e), tn(e))),
                        HP_DV(nv(6 + e)), acc);
  }
#undef HP_DV
  return acc;
}

// Junction currents of a voxel tagged HP_TAG_PMJ (Purkinje potentials from
// Wpk) added to acc; DIAG as in stencil_sum.
template <bool DIAG>
__device__ __forceinline__ float pmj_sum(const MonoArgs& a, float acc, float Vc, int64_t slot,
                                         const float* __restrict__ Wpk) {
  const int r = a.pmj_row[slot];
  for (int q = a.pmj_ptr[r]; q < a.pmj_ptr[r + 1]; ++q)
    acc = __fmaf_rn(a.pmj_coef[q], DIAG ? -1.0f : __fsub_rn(Wpk[a.pmj_pk[q]], Vc), acc);
  return acc;
}

// Neighbour offset q (stencil_sum order) in a tile with strides SI (i), SJ
// (j), 1 (k).
template <int SI, int SJ>
__host__ __device__ constexpr int stencil_off(int q) {
  return q == 0    ? SI
         : q == 1  ? -SI
         : q == 2  ? SJ
         : q == 3  ? -SJ
         : q == 4  ? 1
         : q == 5  ? -1
         : q == 6  ? SI + SJ
         : q == 7  ? -SI - SJ
         : q == 8  ? SI - SJ
         : q == 9  ? -SI + SJ
         : q == 10 ? SI + 1
         : q == 11 ? -SI - 1
         : q == 12 ? SI - 1
         : q == 13 ? -SI + 1
         : q == 14 ? SJ + 1
         : q == 15 ? -SJ - 1
         : q == 16 ? SJ - 1
                   : -SJ + 1;
}

// Stencil sum of one voxel, sum_j coef_ij (W_j - W_i) including its junction
// currents (Purkinje potentials from Wpk), from shared tiles with strides SI
// (i), SJ (j), 1 (k); face weights and off-diagonal tensor components are
// three tiles each, NS floats apart.
template <int SI, int SJ, int NS, bool ANISO, bool DIAG = false>
__device__ __forceinline__ float stencil_acc(const MonoArgs& a, const float* tV, const float* tW,
                                             const float* tD, int c, uint32_t tag, int64_t slot,
                                             const float* __restrict__ Wpk) {
  const float Vc = DIAG ? 0.0f : tV[c];
  float acc = stencil_sum<ANISO, DIAG>(
      a.iso_coef, tag, Vc, [&](int q) { return tV[c + stencil_off<SI, SJ>(q)]; },
      [&](int f) {
        // face weights live on the lower voxel of each face
        return tW[(f >> 1) * NS + c - ((f & 1) ? (f == 1 ? SI : (f == 3 ? SJ : 1)) : 0)];
      },
      [&](int e) { return tD[(e >> 2) * NS + c]; },
      [&](int e) { return tD[(e >> 2) * NS + c + stencil_off<SI, SJ>(6 + e)]; });
  if (tag & HP_TAG_PMJ) acc = pmj_sum<DIAG>(a, acc, Vc, slot, Wpk);
  return acc;
}

// Diffusion half of one voxel (explicit step): V = clamp(W + sum coef (W_j - W)).
template <int SI, int SJ, int NS, bool ANISO>
__device__ __forceinline__ float diffuse(const MonoArgs& a, const float* tV, const float* tW,
                                         const float* tD, int c, uint32_t tag, int64_t slot,
                                         bool odd) {
  const float acc = stencil_acc<SI, SJ, NS, ANISO>(a, tV, tW, tD, c, tag, slot,
                                                   odd ? a.pk_Vs1 : a.pk_Vs0);
  return fminf(fmaxf(__fadd_rn(tV[c], acc), -150.0f), 80.0f);
}

// Outputs of a tissue voxel once V_{i+1} = Vn is known: the
// threshold-crossing test against V_i = Vprev, Vpost and the Vm / surface
// snapshots of step i.
__device__ __forceinline__ void voxel_outputs(const MonoArgs& a, int64_t slot, uint32_t tag,
                                              float Vn, float Vprev, int64_t step,
                                              int64_t vm_frame, int64_t anim_frame) {
  // threshold crossings between the snapshots labelled t_{i-1} and t_i
  if (step >= 1) {
    const bool was_act = Vprev >= a.act_thr, is_act = Vn >= a.act_thr;
    const bool was_dea = Vprev >= a.deact_thr, is_dea = Vn >= a.deact_thr;
    if ((!was_act && is_act) || (was_dea && !is_dea)) {
      const float t0 = (float)((double)(step - 1) * a.dt_d);
      const float t1 = (float)((double)step * a.dt_d);
      if (!was_act && is_act)
        record_event(a.act_t, a.act_n, slot, a.n_slots, a.max_events, a.act_thr, Vprev, Vn, t0,
                     t1);
      if (was_dea && !is_dea)
        record_event(a.deact_t, a.deact_n, slot, a.n_slots, a.max_events, a.deact_thr, Vprev,
                     Vn, t0, t1);
    }
  }
  a.Vpost[slot] = Vn;
  if (vm_frame >= 0) a.vm_snap[vm_frame * a.n_myo + a.node_of_slot[slot]] = Vn;
  if ((tag & HP_TAG_SURF) && anim_frame >= 0)
    a.surf_frames[anim_frame * a.n_surf + a.surf_of_slot[slot]] = Vn;
}

// Ionic half of step istep of a tissue voxel on V = Vn: stores the state and
// W_{istep} = Vn + dt/Cm (-Iion Cm + Istim).
__device__ __forceinline__ void voxel_ionic(const MonoArgs& a, int64_t slot, uint32_t tag, int ph,
                                            float Vn, CellState& cs, int64_t istep, int var,
                                            float* __restrict__ Wout) {
  const CellParams cp = pheno_params(ph, a.var_gks[var], a.var_gkr[var]);
  const float Iion = ttp06_step(Vn, cs, a.dt, cp);
#pragma unroll
  for (int v = 0; v < N_STATE; ++v) a.state[(int64_t)v * a.n_slots + slot] = cs.v[v];
  const float Is = stim_current(a, tag >> HP_TAG_STIM_SHIFT, istep, var);
  Wout[slot] = Vn + a.dt_over_Cm * (-(Iion * a.Cm) + Is);
}

// Everything a tissue voxel does once V_{i+1} = Vn is known (mode 0):
// outputs of step i, then the ionic half of step i+1.  Mode 1 (prologue)
// runs only the ionic half of step 0 on Vn = V_0.
__device__ __forceinline__ void voxel_finish(const MonoArgs& a, int64_t slot, uint32_t tag,
                                             int ph, float Vn, float Vprev, CellState& cs,
                                             int64_t step, int mode, int64_t vm_frame,
                                             int64_t anim_frame, int var, float* Wout) {
  int64_t istep = 0;
  if (mode == 0) {
    voxel_outputs(a, slot, tag, Vn, Vprev, step, vm_frame, anim_frame);
    istep = step + 1;
  }
  voxel_ionic(a, slot, tag, ph, Vn, cs, istep, var, Wout);
}

// Blocks per SM the register budget is sized for (8 x 128 threads -> 64 regs).
template <int BV>
struct MinBlocks {
  static constexpr int value = BV <= 128 ? 8 : (BV <= 256 ? 4 : 2);
};

// One brick per CTA, thread per voxel, halo tiles gathered with plain loads.
// Used for the prologue (mode 1) and where the pipelined kernel does not fit.
template <int BI, int BJ, int BK, bool ANISO>
__global__ void __launch_bounds__(BI * BJ * BK, MinBlocks<BI * BJ * BK>::value)
mono_step_kernel(MonoArgs a, int step_off, int mode) {
  using G = TileGeom<BI, BJ, BK>;
  constexpr int BV = G::BV, SI = G::SI, SJ = G::SJ;
  const int64_t step = *a.d_step + step_off;
  const int tid = threadIdx.x;
  if ((int)blockIdx.x >= a.n_bricks) {
    const int p = ((int)blockIdx.x - a.n_bricks) * BV + tid;
    if (p < a.n_pk) purkinje_part(a, p, step, mode);
    return;
  }
  const int b = blockIdx.x;
  const bool odd = step & 1;
  const float* __restrict__ Win = odd ? a.Vs1 : a.Vs0;
  float* __restrict__ Wout = mode == 0 ? (odd ? a.Vs0 : a.Vs1) : a.Vs0;

  __shared__ int nb27[27];
  __shared__ int64_t s_vm_frame, s_anim_frame;
  __shared__ float tV[G::N];
  __shared__ float tW[ANISO ? 3 * G::N : 1];
  __shared__ float tD[ANISO ? 3 * G::N : 1];
  if (tid < 27) nb27[tid] = a.nbr[(int64_t)b * 27 + tid];
  if (tid == 32) {
    // per-step output decisions, once per block (64-bit modulo is costly)
    s_vm_frame = (a.vm_every > 0 && step % a.vm_every == 0) ? step / a.vm_every : -1;
    s_anim_frame = (a.frame_every > 0 && step % a.frame_every == 0) ? step / a.frame_every : -1;
  }
  // issue this voxel's own loads first so their latency overlaps the halo
  // loads and the stencil: tag, previous post-diffusion V, 18 TTP06 states
  const int64_t slot = (int64_t)b * BV + tid;
  const uint32_t tag = a.tag[slot];
  const float Vprev = a.Vpost[slot];
  CellState cs;
#pragma unroll
  for (int v = 0; v < N_STATE; ++v) cs.v[v] = a.state[(int64_t)v * a.n_slots + slot];
  __syncthreads();
  if (mode == 0) {
    load_region<BI, BJ, BK, -1, BI + 1, -1, BJ + 1, -1, BK + 1>(tV, Win, nb27, tid);
    if constexpr (ANISO) {
      const int64_t ns = a.n_slots;
      load_region<BI, BJ, BK, -1, BI, 0, BJ, 0, BK>(tW, a.wface, nb27, tid);
      load_region<BI, BJ, BK, 0, BI, -1, BJ, 0, BK>(tW + G::N, a.wface + ns, nb27, tid);
      load_region<BI, BJ, BK, 0, BI, 0, BJ, -1, BK>(tW + 2 * G::N, a.wface + 2 * ns, nb27, tid);
      load_region<BI, BJ, BK, -1, BI + 1, -1, BJ + 1, 0, BK>(tD, a.doff, nb27, tid);
      load_region<BI, BJ, BK, -1, BI + 1, 0, BJ, -1, BK + 1>(tD + G::N, a.doff + ns, nb27, tid);
      load_region<BI, BJ, BK, 0, BI, -1, BJ + 1, -1, BK + 1>(tD + 2 * G::N, a.doff + 2 * ns, nb27, tid);
    }
  }
  __syncthreads();

  const int ph = tag & HP_TAG_PHENO_MASK;
  if (ph == 0) return;
  float Vn = Vprev;
  if (mode == 0) {
    const int li = tid / (BJ * BK), lj = (tid / BK) % BJ, lk = tid % BK;
    const int c = (li + 1) * SI + (lj + 1) * SJ + (lk + 1);
    Vn = diffuse<SI, SJ, G::N, ANISO>(a, tV, tW, tD, c, tag, slot, odd);
  }
  const int var = a.brick_variant ? a.brick_variant[b] : 0;
  voxel_finish(a, slot, tag, ph, Vn, Vprev, cs, step, mode, s_vm_frame, s_anim_frame, var, Wout);
}

// ---------------------------------------------------------------------------
// Pipelined persistent step (mode 0).
//
// Each CTA walks the work items blockIdx.x, blockIdx.x + gridDim.x, ...
// (items [0, n_bricks) are bricks, the rest chunks of BV Purkinje nodes).
// While it computes one brick, the data of its next brick -- the W tile with
// its one-voxel halo, for the 19-point operator the face-weight and
// off-diagonal tiles, the 18 TTP06 states, the tag and V_i -- streams into
// the other shared-memory stage with cp.async, so HBM latency is hidden
// behind the TTP06 arithmetic instead of being exposed once per brick.
// Interior rows move as 16-byte copies; the halo elements follow a per-shape
// copy table built on the host (tile position, field, neighbour direction,
// offset in that brick), with zeros where the neighbour brick is absent.
//
// Tile layout in shared memory: k rows of RK = round_up(BK + 2, 4) floats,
// local (li, lj, lk) at 4 + ((lj + 1) * TI + (li + 1)) * RK + lk, so every
// interior row starts on a 16-byte boundary and lk = -1 of a row sits in the
// previous row's padding.  Rows are ordered with i inner: a warp covers
// consecutive slots (fixed li, several lj, all lk), and the j stride TI * RK
// is an odd multiple of the row's width modulo the 32 banks for every
// compiled shape (72, 120 or 80 floats), so the warp's k-rows fall on
// disjoint banks when the stencil reads them.
template <int BI, int BJ, int BK>
struct PipeGeom {
  static constexpr int TI = BI + 2, TJ = BJ + 2, RK = ((BK + 2 + 3) / 4) * 4;
  static constexpr int NT = TI * TJ * RK + 4;  // floats per tile (multiple of 4)
  static constexpr int SI = RK, SJ = TI * RK;
  static constexpr int BV = BI * BJ * BK;
  __host__ __device__ static constexpr int pos(int li, int lj, int lk) {
    return 4 + ((lj + 1) * TI + (li + 1)) * RK + lk;
  }
};

template <int BI, int BJ, int BK, bool ANISO>
struct PipeStage {
  using G = PipeGeom<BI, BJ, BK>;
  static constexpr int NF = ANISO ? 7 : 1;             // staged tiles
  static constexpr int ST = NF * G::NT;                // 18 x BV states
  static constexpr int TAG = ST + N_STATE * G::BV;     // BV tags
  static constexpr int VP = TAG + G::BV;               // BV previous V
  static constexpr int FLOATS = VP + G::BV;
  static constexpr int NCHUNK = (N_STATE + 2) * G::BV / 4;  // 16-byte own-brick copies
};

// halo copy table entry: tile position | field << 11 | direction << 14 |
// offset << 19 | chunk << 31; a chunk entry moves 4 consecutive floats of a
// k-row (16 bytes, both ends 16-byte aligned), otherwise one float
constexpr int HALO_POS_BITS = 11;
constexpr uint32_t HALO_CHUNK = 1u << 31;

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                   (uint32_t)__cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(
                   (uint32_t)__cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
// waits until at most N of this thread's most recent groups are pending
template <int N>
__device__ __forceinline__ void cp_async_wait_pending() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int BI, int BJ, int BK, bool ANISO>
__device__ __forceinline__ void pipe_issue(const MonoArgs& a, float* stage, const uint32_t* tab,
                                           int n_halo, const int* nb27, int b, const float* Win,
                                           int tid) {
  using G = PipeGeom<BI, BJ, BK>;
  using P = PipeStage<BI, BJ, BK, ANISO>;
  constexpr int BV = G::BV;
  const int64_t ns = a.n_slots;
  const int64_t base = (int64_t)b * BV;
  // own brick: 18 states, tag, V_i (contiguous BV-float runs)
  for (int q = tid; q < P::NCHUNK; q += BV) {
    const int f = q / (BV / 4), o = (q % (BV / 4)) * 4;
    const float* src = f < N_STATE ? a.state + (int64_t)f * ns
                                   : (f == N_STATE ? (const float*)a.tag : a.Vpost);
    cp_async16(stage + P::ST + f * BV + o, src + base + o);
  }
  // own brick rows of the staged tiles
  for (int q = tid; q < P::NF * (BV / 4); q += BV) {
    const int f = q / (BV / 4), o = (q % (BV / 4)) * 4;
    const int gi = o / (BJ * BK), gj = (o / BK) % BJ, gk = o % BK;
    const float* src = f == 0 ? Win : (f < 4 ? a.wface + (f - 1) * ns : a.doff + (f - 4) * ns);
    cp_async16(stage + f * G::NT + G::pos(gi, gj, gk), src + base + o);
  }
  // halo elements
  for (int e = tid; e < n_halo; e += BV) {
    const uint32_t t = tab[e];
    const int pos = t & ((1u << HALO_POS_BITS) - 1), f = (t >> 11) & 7, dir = (t >> 14) & 31,
              off = (int)((t >> 19) & 0xFFFu);
    const int nb = nb27[dir];
    float* dst = stage + f * G::NT + pos;
    if (nb >= 0) {
      const float* src = f == 0 ? Win : (f < 4 ? a.wface + (f - 1) * ns : a.doff + (f - 4) * ns);
      if (t & HALO_CHUNK)
        cp_async16(dst, src + (int64_t)nb * BV + off);
      else
        cp_async4(dst, src + (int64_t)nb * BV + off);
    } else if (t & HALO_CHUNK) {
      *(float4*)dst = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    } else {
      *dst = 0.0f;
    }
  }
}

template <int BV>
struct PipeMinBlocks {
  static constexpr int value = BV <= 128 ? 4 : (BV <= 256 ? 2 : 1);
};

template <int BI, int BJ, int BK, bool ANISO>
__global__ void __launch_bounds__(BI * BJ * BK, PipeMinBlocks<BI * BJ * BK>::value)
mono_pipe_kernel(MonoArgs a, int step_off) {
  using G = PipeGeom<BI, BJ, BK>;
  using P = PipeStage<BI, BJ, BK, ANISO>;
  constexpr int BV = G::BV;
  extern __shared__ __align__(16) float smem[];
  float* stages = smem;                                       // 2 x FLOATS
  uint32_t* tab = (uint32_t*)(smem + 2 * P::FLOATS);          // n_halo
  int* ring = (int*)(tab + ((a.n_halo + 3) & ~3));            // 2 x 27 neighbour lists
  __shared__ int64_t s_vm_frame, s_anim_frame;

  const int tid = threadIdx.x;
  const int64_t step = *a.d_step + step_off;
  const bool odd = step & 1;
  const float* __restrict__ Win = odd ? a.Vs1 : a.Vs0;
  float* __restrict__ Wout = odd ? a.Vs0 : a.Vs1;
  const int G_ = gridDim.x;
  const int n_items = a.n_bricks + (a.n_pk + BV - 1) / BV;

  for (int e = tid; e < a.n_halo; e += BV) tab[e] = a.halo_tab[e];
  if (tid == 0) {
    s_vm_frame = (a.vm_every > 0 && step % a.vm_every == 0) ? step / a.vm_every : -1;
    s_anim_frame = (a.frame_every > 0 && step % a.frame_every == 0) ? step / a.frame_every : -1;
  }
  int cur = blockIdx.x;
  if (cur < a.n_bricks && tid < 27) ring[tid] = a.nbr[(int64_t)cur * 27 + tid];
  __syncthreads();
  if (cur < a.n_bricks) {
    pipe_issue<BI, BJ, BK, ANISO>(a, stages, tab, a.n_halo, ring, cur, Win, tid);
    const int nx = cur + G_;
    if (nx < a.n_bricks && tid < 27) cp_async4(ring + 27 + tid, a.nbr + (int64_t)nx * 27 + tid);
  }
  cp_async_commit();

  for (int n = 0; cur < n_items; ++n, cur += G_) {
    cp_async_wait_all();
    __syncthreads();
    const int nxt = cur + G_;
    if (nxt < a.n_bricks) {
      pipe_issue<BI, BJ, BK, ANISO>(a, stages + ((n + 1) & 1) * P::FLOATS, tab, a.n_halo,
                                    ring + ((n + 1) & 1) * 27, nxt, Win, tid);
      const int nn = nxt + G_;
      if (nn < a.n_bricks && tid < 27)
        cp_async4(ring + (n & 1) * 27 + tid, a.nbr + (int64_t)nn * 27 + tid);
    }
    cp_async_commit();
    if (cur < a.n_bricks) {
      const float* st = stages + (n & 1) * P::FLOATS;
      const uint32_t tag = ((const uint32_t*)(st + P::TAG))[tid];
      const int ph = tag & HP_TAG_PHENO_MASK;
      if (ph != 0) {
        const int64_t slot = (int64_t)cur * BV + tid;
        const int li = tid / (BJ * BK), lj = (tid / BK) % BJ, lk = tid % BK;
        const float Vn = diffuse<G::SI, G::SJ, G::NT, ANISO>(
            a, st, st + G::NT, st + 4 * G::NT, G::pos(li, lj, lk), tag, slot, odd);
        CellState cs;
#pragma unroll
        for (int v = 0; v < N_STATE; ++v) cs.v[v] = st[P::ST + v * BV + tid];
        const float Vprev = st[P::VP + tid];
        const int var = a.brick_variant ? a.brick_variant[cur] : 0;
        voxel_finish(a, slot, tag, ph, Vn, Vprev, cs, step, 0, s_vm_frame, s_anim_frame, var,
                     Wout);
      }
    } else {
      const int p = (cur - a.n_bricks) * BV + tid;
      if (p < a.n_pk) purkinje_part(a, p, step, 0);
    }
    __syncthreads();
  }
  cp_async_wait_all();
}

// ---------------------------------------------------------------------------
// Crank-Nicolson diffusion half (theta > 0).
//
// The reference solves (Cm/dt) V_{i+1} - theta L V_{i+1} = (Cm/dt) W_i +
// (1 - theta) L W_i by Jacobi-preconditioned BiCGSTAB from V_{i+1} = W_i
// (purkinje_myocardium_pipeline.py:662-754, :1383-1391; anisotropic solver
// :1784-1790), then clamps to [-150, 80].  With the coefficients pre-scaled
// by dt / (Cm Ai) the system is M x = W + (1 - theta) Lh W, M = I - theta Lh.
// Lh = D^-1 K with K symmetric and D = diag(Ai) (Ai_M on tissue, Ai_P on
// Purkinje nodes), so M is self-adjoint in the inner product weighted by
// Ai / Ai_M: this solver runs Jacobi-preconditioned CG in that inner product
// (weight 1 on tissue slots, pk_weight = Ai_P / Ai_M on Purkinje nodes).
// The stopping rule is the reference's: unweighted ||r|| <= tol ||rhs||.
//
// CG vectors are [slots | Purkinje nodes] of length n_slots + n_pk, FP32;
// dot products are FP64 with deterministic last-block grid reductions.  The
// warm-start residual rhs - M W equals Lh W, so one stencil pass gives the
// initial residual, the norm of the right-hand side and the first direction.
// Every iteration kernel returns at once when the done flag is set, so the
// host may enqueue iterations in chunks and test the flag between chunks.
enum CnScal : int { CN_BB = 0, CN_RZ, CN_PQ, CN_ALPHA, CN_BETA, CN_RR, N_CN_SCAL };
enum CnIScal : int { CI_DONE = 0, CI_ITER, CI_TOTAL, CI_SOLVES, CI_UNCONV, CI_BREAK, CI_LOOP,
                     N_CN_ISCAL };
constexpr int CN_TB = 256;   // threads of the vector kernels
constexpr int CN_NPART = 4;  // partials per block

struct CnArgs {
  int64_t n;             // n_slots + n_pk
  float theta, omt;      // theta and 1 - theta
  float pk_weight;       // Ai_P / Ai_M
  double tol2;           // squared relative tolerance
  int32_t max_iter;
  float* x;
  float* r;
  float* p;
  float* q;
  float* dinv;           // 1 / diag(M); 0 on padding slots
  double* part;          // grid x CN_NPART partial sums
  double* scal;
  int32_t* iscal;
  unsigned int* ticket;
};

// Block-reduces NV sums into part[blockIdx.x]; true in the last block to
// arrive, whose threads then all hold the grid totals in tot (summed in
// block order, so the result does not depend on scheduling).
template <int NT, int NV>
__device__ bool cn_reduce_last(double (&v)[NV], const CnArgs& c, double (&tot)[NV]) {
  __shared__ double sh[NT / 32][NV];
  __shared__ double sh2[NT][NV];
  __shared__ bool am_last;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double w = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) w += __shfl_down_sync(0xffffffffu, w, o);
    if (lane == 0) sh[wid][k] = w;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double s = sh[0][k];
      for (int w = 1; w < NT / 32; ++w) s += sh[w][k];
      c.part[(int64_t)blockIdx.x * CN_NPART + k] = s;
    }
    __threadfence();
    am_last = atomicAdd(c.ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!am_last) return false;
  __threadfence();
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = 0.0;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += NT) {
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] += ((volatile double*)c.part)[(int64_t)b * CN_NPART + k];
  }
#pragma unroll
  for (int k = 0; k < NV; ++k) sh2[threadIdx.x][k] = v[k];
  __syncthreads();
  for (int s = NT / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
#pragma unroll
      for (int k = 0; k < NV; ++k) sh2[threadIdx.x][k] += sh2[threadIdx.x + s][k];
    }
    __syncthreads();
  }
#pragma unroll
  for (int k = 0; k < NV; ++k) tot[k] = sh2[0][k];
  if (threadIdx.x == 0) *c.ticket = 0u;
  return true;
}

// ---------------------------------------------------------------------------
// Split step: two launches per step over the same arrays.
//
// mono_diffuse_kernel (one CTA per brick, plus CTAs of BV Purkinje nodes)
// forms V_{i+1} from W_i and its halo, records the crossings and snapshots of
// step i and stores V_{i+1} in Vpost.  mono_ionic_kernel then runs the ionic
// half of step i+1 with one thread per tissue slot, taken from the compact
// list active_slot, so padding slots of partially filled bricks occupy no
// lane, and without shared memory or barriers, so it runs at full occupancy.
// Both do the fused kernels' arithmetic in the same order: results are
// bit-identical to theirs.
// Halo copy-table entries per thread of the diffusion kernel (held in
// registers for the whole launch).  Rows of a face or ij-edge outside the
// brick in i or j move as BK/4 16-byte chunks, k-face and k-edge elements
// one by one.
template <int BI, int BJ, int BK, bool ANISO>
struct DiffHalo {
  static constexpr int BV = BI * BJ * BK, Q = BK / 4;
  static constexpr int W = ANISO ? 2 * (BI + BJ + 2) * Q + 2 * BI * BJ + 4 * (BI + BJ)
                                 : 2 * (BI + BJ) * Q + 2 * BI * BJ;
  // face weights (-i, -j, -k faces) and the three off-diagonal tiles
  static constexpr int A = (BJ + BI) * Q + BI * BJ + (2 * BJ + 2 * BI + 4) * Q +
                           (2 * BJ * Q + 2 * BI * BJ + 4 * BJ) + (2 * BI * Q + 2 * BI * BJ + 4 * BI);
  static constexpr int N = ANISO ? W + A : W;
  static constexpr int PER_THREAD = (N + BV - 1) / BV;
};

// Shared-memory stage of the diffusion kernel: the staged tiles, then the
// brick's tags and V_i.  NS stages are in flight or in use per CTA (the
// bricks of NS - 1 stages stream in while one is computed), and the
// neighbour lists of the next RING bricks ride along in the same groups.
#ifndef HP_DIFF_STAGES
#define HP_DIFF_STAGES 2
#endif
template <int BI, int BJ, int BK, bool ANISO>
struct DiffStage {
  using G = PipeGeom<BI, BJ, BK>;
  static constexpr int NS = HP_DIFF_STAGES;
  static constexpr int RING = 2 * NS;
  static constexpr int NF = ANISO ? 7 : 1;
  static constexpr int TAG = NF * G::NT;
  static constexpr int VP = TAG + G::BV;
  static constexpr int FLOATS = VP + G::BV;
  static constexpr int SMEM_FLOATS = NS * FLOATS + 27 * RING;  // + the neighbour-list ring
  static constexpr int NCHUNK = (NF + 2) * G::BV / 4;  // 16-byte own-brick copies
};

// CN operations of the diffusion pass (OP template argument; 0 is the
// explicit step).
constexpr int OP_STEP = 0, OP_CN_START = 1, OP_CN_APPLY = 2;

// Last-block scalars of a CN stencil pass (mode OP_CN_START or OP_CN_APPLY)
// from the grid totals: the start of a solve records ||rhs||^2, ||r||^2 and
// <r, z>_w and tests the warm start; an application forms alpha.
__device__ __forceinline__ void cn_pass_scalars(const CnArgs& c, int op, const double (&tot)[3]) {
  if (op == OP_CN_START) {
    c.scal[CN_BB] = tot[0];
    c.scal[CN_RR] = tot[1];
    c.scal[CN_RZ] = tot[2];
    c.iscal[CI_ITER] = 0;
    c.iscal[CI_SOLVES] += 1;
    // converged at the warm start (also a zero right-hand side)
    c.iscal[CI_DONE] = (tot[1] <= c.tol2 * tot[0] || tot[0] == 0.0) ? 1 : 0;
  } else {
    const double pq = tot[0];
    if (!(pq > 0.0) || !isfinite(pq)) {  // breakdown: keep the current x
      c.iscal[CI_BREAK] += 1;
      c.iscal[CI_DONE] = 1;
    } else {
      c.scal[CN_PQ] = pq;
      c.scal[CN_ALPHA] = c.scal[CN_RZ] / pq;
    }
  }
}

// Persistent diffusion pass over bricks (then chunks of BV Purkinje nodes),
// tiles double-buffered with cp.async.  OP_STEP: the explicit diffusion half
// of the split step (V_{i+1} from W_i, outputs of step i).  OP_CN_START: the
// start of a theta-scheme solve on W_i (x = W, r = Lh W, p = Dinv r and
// their sums).  OP_CN_APPLY: q = p - theta Lh p and <p, q>_w.  The CN
// passes write tissue entries only: padding entries of the CG vectors are
// zero from set-up and stay zero.
template <int BI, int BJ, int BK, bool ANISO, int OP>
__device__ __forceinline__ void diffuse_pass(const MonoArgs a, const CnArgs cn, int step_off) {
  using G = PipeGeom<BI, BJ, BK>;
  using H = DiffHalo<BI, BJ, BK, ANISO>;
  using D = DiffStage<BI, BJ, BK, ANISO>;
  constexpr int BV = G::BV, NF = D::NF, PT = H::PER_THREAD;
  constexpr int QB = BV / 4;  // 16-byte chunks per brick row of one field
  // per-slot fields after the tiles: tag, then V_i (step) or Dinv (start)
  constexpr int NCHUNK = OP == OP_CN_APPLY ? (NF + 1) * BV / 4 : D::NCHUNK;
  constexpr int NS = D::NS, RS = D::RING;
  extern __shared__ __align__(16) float smem[];
  float* stages = smem;                       // NS x FLOATS
  int* ring = (int*)(smem + NS * D::FLOATS);  // RS x 27 neighbour lists
  __shared__ int64_t s_vm_frame, s_anim_frame;
  if (OP == OP_CN_APPLY && cn.iscal[CI_DONE]) return;
  const int64_t step = *a.d_step + step_off;
  const bool odd = step & 1;
  const float* __restrict__ Win = OP == OP_CN_APPLY ? cn.p : (odd ? a.Vs1 : a.Vs0);
  const float* __restrict__ Wpk = OP == OP_CN_APPLY ? cn.p + a.n_slots : (odd ? a.pk_Vs1 : a.pk_Vs0);
  const float* __restrict__ Xtra = OP == OP_STEP ? a.Vpost : cn.dinv;
  const int tid = threadIdx.x;
  const int64_t ns = a.n_slots;
  // this thread's halo copies for the whole launch: stage offset (field tile
  // + position), neighbour direction, source (array + offset in the brick)
  uint32_t hpos[PT], hdir[PT];
  const float* hsrc[PT];
#pragma unroll
  for (int q = 0; q < PT; ++q) {
    const int e = tid + q * BV;
    const uint32_t t = e < a.n_halo ? a.halo_tab[e] : 0u;
    const int f = (t >> 11) & 7;
    hpos[q] = e < a.n_halo ? (uint32_t)(f * G::NT + (int)(t & ((1u << HALO_POS_BITS) - 1)))
                           : 0xFFFFFFFFu;
    hdir[q] = ((t >> 14) & 31) | ((t & HALO_CHUNK) ? 32u : 0u);
    hsrc[q] = e >= a.n_halo ? Win
                            : (f == 0 ? Win : (f < 4 ? a.wface + (f - 1) * ns : a.doff + (f - 4) * ns)) +
                                  ((t >> 19) & 0xFFFu);
  }
  auto issue = [&](float* st, const int* nb27, int b) {
    const int64_t base = (int64_t)b * BV;
#pragma unroll
    for (int k = 0; k < (NCHUNK + BV - 1) / BV; ++k) {
      const int q = tid + k * BV;
      if (q < NCHUNK) {
        const int f = q / QB, o = (q % QB) * 4;
        const float* src = f == 0    ? Win
                           : f < NF  ? (f < 4 ? a.wface + (f - 1) * ns : a.doff + (f - 4) * ns)
                           : f == NF ? (const float*)a.tag
                                     : Xtra;
        float* dst = f < NF ? st + f * G::NT + G::pos(o / (BJ * BK), (o / BK) % BJ, o % BK)
                            : st + D::TAG + (f - NF) * BV + o;
        cp_async16(dst, src + base + o);
      }
    }
#pragma unroll
    for (int q = 0; q < PT; ++q) {
      if (hpos[q] != 0xFFFFFFFFu) {
        const int nb = nb27[hdir[q] & 31];
        const bool chunk = hdir[q] & 32;
        if (nb >= 0) {
          if (chunk)
            cp_async16(st + hpos[q], hsrc[q] + (int64_t)nb * BV);
          else
            cp_async4(st + hpos[q], hsrc[q] + (int64_t)nb * BV);
        } else if (chunk) {
          *(float4*)(st + hpos[q]) = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        } else {
          st[hpos[q]] = 0.0f;
        }
      }
    }
  };
  const int li = tid / (BJ * BK), lj = (tid / BK) % BJ, lk = tid % BK;
  const int c = G::pos(li, lj, lk);
  const int G_ = gridDim.x;
  const int n_items = a.n_bricks + (a.n_pk + BV - 1) / BV;
  if (tid == 0) {
    s_vm_frame = (a.vm_every > 0 && step % a.vm_every == 0) ? step / a.vm_every : -1;
    s_anim_frame = (a.frame_every > 0 && step % a.frame_every == 0) ? step / a.frame_every : -1;
  }
  double v[3] = {0.0, 0.0, 0.0};  // CN sums
  // item m of this CTA is blockIdx.x + m G_, staged in stage m % NS; its
  // neighbour list sits in ring slot m % RS, fetched together with item
  // m - (NS - 1) (the first NS - 1 lists are loaded directly), so it is
  // complete by the time item m is issued
  int cur = blockIdx.x;
#pragma unroll
  for (int m = 0; m < NS - 1; ++m) {
    const int it = cur + m * G_;
    if (it < a.n_bricks && tid < 27) ring[(m % RS) * 27 + tid] = a.nbr[(int64_t)it * 27 + tid];
  }
  __syncthreads();
#pragma unroll
  for (int m = 0; m < NS - 1; ++m) {
    const int it = cur + m * G_;
    if (it < a.n_bricks) {
      issue(stages + m * D::FLOATS, ring + (m % RS) * 27, it);
      const int ahead = it + (NS - 1) * G_;
      if (ahead < a.n_bricks && tid < 27)
        cp_async4(ring + ((m + NS - 1) % RS) * 27 + tid, a.nbr + (int64_t)ahead * 27 + tid);
    }
    cp_async_commit();
  }
  for (int n = 0; cur < n_items; ++n, cur += G_) {
    cp_async_wait_pending<NS - 2>();  // item n has landed
    __syncthreads();
    const int m = n + NS - 1;
    const int it = cur + (NS - 1) * G_;
    if (it < a.n_bricks) {
      issue(stages + (m % NS) * D::FLOATS, ring + (m % RS) * 27, it);
      const int ahead = it + (NS - 1) * G_;
      if (ahead < a.n_bricks && tid < 27)
        cp_async4(ring + ((m + NS - 1) % RS) * 27 + tid, a.nbr + (int64_t)ahead * 27 + tid);
    }
    cp_async_commit();
    if (cur < a.n_bricks) {
      const float* st = stages + (n % NS) * D::FLOATS;
      const uint32_t tag = ((const uint32_t*)(st + D::TAG))[tid];
      if (tag & HP_TAG_PHENO_MASK) {
        const int64_t slot = (int64_t)cur * BV + tid;
        const float* tW = ANISO ? st + G::NT : st;
        const float* tD = ANISO ? st + 4 * G::NT : st;
        if constexpr (OP == OP_STEP) {
          const float Vn = diffuse<G::SI, G::SJ, G::NT, ANISO>(a, st, tW, tD, c, tag, slot, odd);
          voxel_outputs(a, slot, tag, Vn, st[D::VP + tid], step, s_vm_frame, s_anim_frame);
        } else {
          const float acc = stencil_acc<G::SI, G::SJ, G::NT, ANISO>(a, st, tW, tD, c, tag, slot, Wpk);
          if constexpr (OP == OP_CN_START) {
            const float Wi = st[c], z = st[D::VP + tid] * acc, b = Wi + cn.omt * acc;
            cn.x[slot] = Wi;
            cn.r[slot] = acc;
            cn.p[slot] = z;
            v[0] += (double)b * b;
            v[1] += (double)acc * acc;
            v[2] += (double)acc * z;
          } else {
            const float pi = st[c], qi = pi - cn.theta * acc;
            cn.q[slot] = qi;
            v[0] += (double)pi * qi;
          }
        }
      }
    } else {
      const int p = (cur - a.n_bricks) * BV + tid;
      if (p < a.n_pk) {
        if constexpr (OP == OP_STEP) {
          purkinje_diffuse(a, p, step);
        } else {
          const float acc = purkinje_acc(a, p, Wpk, Win);
          const int64_t e = a.n_slots + p;
          const float w = cn.pk_weight;
          if constexpr (OP == OP_CN_START) {
            const float Wi = Wpk[p], z = cn.dinv[e] * acc, b = Wi + cn.omt * acc;
            cn.x[e] = Wi;
            cn.r[e] = acc;
            cn.p[e] = z;
            v[0] += (double)b * b;
            v[1] += (double)acc * acc;
            v[2] += (double)w * acc * z;
          } else {
            const float pi = Wpk[p], qi = pi - cn.theta * acc;
            cn.q[e] = qi;
            v[0] += (double)w * pi * qi;
          }
        }
      }
    }
    __syncthreads();
  }
  cp_async_wait_all();
  if constexpr (OP != OP_STEP) {
    double tot[3];
    if (cn_reduce_last<BV, 3>(v, cn, tot) && threadIdx.x == 0) cn_pass_scalars(cn, OP, tot);
  }
}

template <int BI, int BJ, int BK, bool ANISO>
__global__ void __launch_bounds__(BI * BJ * BK)
mono_diffuse_kernel(MonoArgs a, int step_off) {
  CnArgs none{};
  diffuse_pass<BI, BJ, BK, ANISO, OP_STEP>(a, none, step_off);
}

// The two CN passes on the persistent diffusion kernel's tiles.
template <int BI, int BJ, int BK, bool ANISO, int OP>
__global__ void __launch_bounds__(BI * BJ * BK) cn_pass_kernel(MonoArgs a, CnArgs c) {
  diffuse_pass<BI, BJ, BK, ANISO, OP>(a, c, 0);
}

constexpr int ION_THREADS = 128;

// The split step keeps the 18 TTP06 states in compact tissue order (index
// i of active_slot, not the slot), so the ionic half's state loads and
// stores are fully coalesced; tag, V and W stay per slot for the stencil.
// mode 1: the prologue, the ionic half of step 0 on V_0 into W_0.
// mode 0: the ionic half of step i+1 on V_{i+1} = Vpost; mode 1: the
// prologue, the ionic half of step 0 on V_0 into W_0; mode 2: the end of a
// theta-scheme step, V_{i+1} = clamp(x) with the outputs of step i recorded
// exactly as the explicit step records them, then the ionic half of step
// i+1 on it.
template <int mode>
__global__ void __launch_bounds__(ION_THREADS, 8) mono_ionic_kernel(MonoArgs a, int step_off) {
  __shared__ int64_t s_vm_frame, s_anim_frame;
  const int64_t step = *a.d_step + step_off;
  if constexpr (mode == 2) {
    if (threadIdx.x == 0) {
      s_vm_frame = (a.vm_every > 0 && step % a.vm_every == 0) ? step / a.vm_every : -1;
      s_anim_frame = (a.frame_every > 0 && step % a.frame_every == 0) ? step / a.frame_every : -1;
    }
    __syncthreads();
  }
  const bool odd = step & 1;
  const int64_t istep = mode == 1 ? 0 : step + 1;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.n_active) {
    const int64_t slot = a.active_slot[i];
    const uint32_t tag = a.tag[slot];
    float Vn;
    if constexpr (mode == 2) {
      Vn = fminf(fmaxf(a.cn_x[slot], -150.0f), 80.0f);
      voxel_outputs(a, slot, tag, Vn, a.Vpost[slot], step, s_vm_frame, s_anim_frame);
    } else {
      Vn = a.Vpost[slot];
    }
    const int64_t na = a.n_active;
    CellState cs;
#pragma unroll
    for (int v = 0; v < N_STATE; ++v) cs.v[v] = a.state[(int64_t)v * na + i];
    const int var = a.brick_variant ? a.brick_variant[slot >> a.bv_shift] : 0;
    const CellParams cp = pheno_params(tag & HP_TAG_PHENO_MASK, a.var_gks[var], a.var_gkr[var]);
    const float Iion = ttp06_step(Vn, cs, a.dt, cp);
#pragma unroll
    for (int v = 0; v < N_STATE; ++v) a.state[(int64_t)v * na + i] = cs.v[v];
    const float Is = stim_current(a, tag >> HP_TAG_STIM_SHIFT, istep, var);
    float* __restrict__ Wout = mode == 1 ? a.Vs0 : (odd ? a.Vs0 : a.Vs1);
    Wout[slot] = Vn + a.dt_over_Cm * (-(Iion * a.Cm) + Is);
  } else {
    const int p = i - a.n_active_pad;
    if (p >= 0 && p < a.n_pk) {
      float Vn;
      if constexpr (mode == 2) {
        Vn = fminf(fmaxf(a.cn_x[a.n_slots + p], -150.0f), 80.0f);
        a.pk_Vpost[p] = Vn;
        if (s_anim_frame >= 0) a.pk_frames[s_anim_frame * (int64_t)a.n_pk + p] = Vn;
      } else {
        Vn = a.pk_Vpost[p];
      }
      purkinje_ionic(a, p, Vn, istep, mode == 1 ? a.pk_Vs0 : (odd ? a.pk_Vs0 : a.pk_Vs1));
    }
  }
}

// Set-up of the theta-scheme solve: the Jacobi inverse dinv = 1 / (1 - theta
// diag Lh) of every tissue slot and Purkinje node (0 on padding slots), from
// the same stencil code with every difference read as -1.  Persistent CTAs
// over bricks, then chunks of BV Purkinje nodes; plain halo loads (it runs
// once per handle).
template <int BI, int BJ, int BK, bool ANISO>
__global__ void __launch_bounds__(BI * BJ * BK) cn_diag_kernel(MonoArgs a, CnArgs c) {
  using G = TileGeom<BI, BJ, BK>;
  constexpr int BV = G::BV, SI = G::SI, SJ = G::SJ;
  const int64_t ns = a.n_slots;
  __shared__ int nb27[27];
  __shared__ float tW[ANISO ? 3 * G::N : 1];
  __shared__ float tD[ANISO ? 3 * G::N : 1];
  const int tid = threadIdx.x;
  const int li = tid / (BJ * BK), lj = (tid / BK) % BJ, lk = tid % BK;
  const int cc = (li + 1) * SI + (lj + 1) * SJ + (lk + 1);
  const int n_items = a.n_bricks + (a.n_pk + BV - 1) / BV;
  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    if (it >= a.n_bricks) {
      const int pn = (it - a.n_bricks) * BV + tid;
      if (pn < a.n_pk)
        c.dinv[ns + pn] = 1.0f / (1.0f - c.theta * purkinje_acc<true>(a, pn, nullptr, nullptr));
      continue;
    }
    __syncthreads();  // the previous brick's tiles are no longer read
    if (tid < 27) nb27[tid] = a.nbr[(int64_t)it * 27 + tid];
    __syncthreads();
    if constexpr (ANISO) {
      load_region<BI, BJ, BK, -1, BI, 0, BJ, 0, BK>(tW, a.wface, nb27, tid);
      load_region<BI, BJ, BK, 0, BI, -1, BJ, 0, BK>(tW + G::N, a.wface + ns, nb27, tid);
      load_region<BI, BJ, BK, 0, BI, 0, BJ, -1, BK>(tW + 2 * G::N, a.wface + 2 * ns, nb27, tid);
      load_region<BI, BJ, BK, -1, BI + 1, -1, BJ + 1, 0, BK>(tD, a.doff, nb27, tid);
      load_region<BI, BJ, BK, -1, BI + 1, 0, BJ, -1, BK + 1>(tD + G::N, a.doff + ns, nb27, tid);
      load_region<BI, BJ, BK, 0, BI, -1, BJ + 1, -1, BK + 1>(tD + 2 * G::N, a.doff + 2 * ns, nb27, tid);
    }
    __syncthreads();
    const int64_t slot = (int64_t)it * BV + tid;
    const uint32_t tag = a.tag[slot];
    c.dinv[slot] = (tag & HP_TAG_PHENO_MASK)
                       ? 1.0f / (1.0f - c.theta * stencil_acc<SI, SJ, G::N, ANISO, true>(
                                                  a, nullptr, tW, tD, cc, tag, slot, nullptr))
                       : 0.0f;
  }
}

// x += alpha p, r -= alpha q; sums ||r||^2 and <r, Dinv r>_w; the last block
// takes beta and the stopping decision.
__global__ void __launch_bounds__(CN_TB) cn_update_kernel(CnArgs c, int64_t ns) {
  if (c.iscal[CI_DONE]) return;
  const float alpha = (float)c.scal[CN_ALPHA];
  double v[2] = {0.0, 0.0};
  for (int64_t e = blockIdx.x * (int64_t)CN_TB + threadIdx.x; e < c.n;
       e += (int64_t)gridDim.x * CN_TB) {
    const float xi = c.x[e] + alpha * c.p[e];
    const float ri = c.r[e] - alpha * c.q[e];
    c.x[e] = xi;
    c.r[e] = ri;
    const float z = c.dinv[e] * ri;
    v[0] += (double)ri * ri;
    v[1] += (double)(e < ns ? 1.0f : c.pk_weight) * ri * z;
  }
  double tot[2];
  if (!cn_reduce_last<CN_TB, 2>(v, c, tot)) return;
  if (threadIdx.x != 0) return;
  const int it = c.iscal[CI_ITER] + 1;
  c.iscal[CI_ITER] = it;
  c.iscal[CI_TOTAL] += 1;
  c.scal[CN_RR] = tot[0];
  const double rz_old = c.scal[CN_RZ];
  c.scal[CN_BETA] = rz_old > 0.0 ? tot[1] / rz_old : 0.0;
  c.scal[CN_RZ] = tot[1];
  if (tot[0] <= c.tol2 * c.scal[CN_BB]) {
    c.iscal[CI_DONE] = 1;
  } else if (it >= c.max_iter || !isfinite(tot[0])) {
    c.iscal[CI_UNCONV] += 1;
    c.iscal[CI_DONE] = 1;
  }
}

// p = Dinv r + beta p.
__global__ void __launch_bounds__(CN_TB) cn_dir_kernel(CnArgs c) {
  if (c.iscal[CI_DONE]) return;
  const float beta = (float)c.scal[CN_BETA];
  for (int64_t e = blockIdx.x * (int64_t)CN_TB + threadIdx.x; e < c.n;
       e += (int64_t)gridDim.x * CN_TB)
    c.p[e] = c.dinv[e] * c.r[e] + beta * c.p[e];
}

// Loop condition of a solve captured in a CUDA graph (a conditional WHILE
// node): before the loop (init) "not yet converged", after each iteration
// "not converged and fewer than max_iter iterations".  Its own counter
// bounds the loop whatever the other kernels do.
__global__ void cn_cond_kernel(cudaGraphConditionalHandle hd, CnArgs c, int init) {
  int n = 0;
  if (init)
    c.iscal[CI_LOOP] = 0;
  else
    n = ++c.iscal[CI_LOOP];
  cudaGraphSetConditional(hd, (!c.iscal[CI_DONE] && n < c.max_iter) ? 1u : 0u);
}

// Host: halo copy table of the pipelined and split-diffusion kernels for
// one brick shape: the union of the tile elements the stencil reads, minus
// the brick's own voxels (the 7-point operator reads face neighbours only,
// the 19-point one faces and edges, neither the cube's corners).
template <int BI, int BJ, int BK>
static std::vector<uint32_t> pipe_halo_table(bool aniso) {
  using G = PipeGeom<BI, BJ, BK>;
  static_assert(BK % 4 == 0, "k rows move as 16-byte chunks");
  std::vector<uint32_t> t;
  auto entry = [&](int f, int li, int lj, int lk, bool chunk) {
    const int di = li < 0 ? -1 : (li >= BI ? 1 : 0);
    const int dj = lj < 0 ? -1 : (lj >= BJ ? 1 : 0);
    const int dk = lk < 0 ? -1 : (lk >= BK ? 1 : 0);
    const int gi = li - di * BI, gj = lj - dj * BJ, gk = lk - dk * BK;
    const uint32_t off = (uint32_t)((gi * BJ + gj) * BK + gk);
    const uint32_t dir = (uint32_t)((di + 1) * 9 + (dj + 1) * 3 + (dk + 1));
    t.push_back((uint32_t)G::pos(li, lj, lk) | ((uint32_t)f << 11) | (dir << 14) | (off << 19) |
                (chunk ? HALO_CHUNK : 0u));
  };
  auto needed = [&](int li, int lj, int lk) {
    const int n_out = (li < 0 || li >= BI) + (lj < 0 || lj >= BJ) + (lk < 0 || lk >= BK);
    return n_out > 0 && n_out <= (aniso ? 2 : 1);
  };
  auto region = [&](int f, int i0, int i1, int j0, int j1, int k0, int k1) {
    for (int li = i0; li < i1; ++li)
      for (int lj = j0; lj < j1; ++lj) {
        const bool side = li < 0 || li >= BI || lj < 0 || lj >= BJ;
        // the interior part of a k-row outside the brick in i or j is
        // contiguous in the neighbour brick: 16-byte chunks
        const bool rows = side && k0 <= 0 && k1 >= BK && needed(li, lj, 0);
        for (int lk = k0; lk < k1; ++lk) {
          if (rows && lk >= 0 && lk < BK) {
            if (lk % 4 == 0) entry(f, li, lj, lk, true);
            continue;
          }
          if (needed(li, lj, lk)) entry(f, li, lj, lk, false);
        }
      }
  };
  region(0, -1, BI + 1, -1, BJ + 1, -1, BK + 1);
  if (aniso) {
    region(1, -1, BI, 0, BJ, 0, BK);
    region(2, 0, BI, -1, BJ, 0, BK);
    region(3, 0, BI, 0, BJ, -1, BK);
    region(4, -1, BI + 1, -1, BJ + 1, 0, BK);
    region(5, -1, BI + 1, 0, BJ, -1, BK + 1);
    region(6, 0, BI, -1, BJ + 1, -1, BK + 1);
  }
  return t;
}

__global__ void init_cells_kernel(float* state, float* Vpost, int64_t n, float v0) {
  // resting state, gpu_ttp06.py:150-169
  const float init[N_STATE] = {138.4f, 10.355f, 0.00013f, 0.00448f, 0.476f, 0.0087f,
                               0.00155f, 0.7573f, 0.7225f, 3.164e-5f, 0.8009f, 0.9778f,
                               0.9953f, 0.3212f, 2.235e-8f, 3.715f, 0.9068f, 0.00036f};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int v = 0; v < N_STATE; ++v) state[v * n + i] = init[v];
    Vpost[i] = v0;
  }
}

__global__ void fill_kernel(float* p, int64_t n, float v) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    p[i] = v;
}

__global__ void advance_kernel(int64_t* d_step, int64_t n) { *d_step += n; }

typedef void (*StepFn)(MonoArgs, int, int);
typedef void (*CnFn)(MonoArgs, CnArgs);
typedef void (*CnPassFn)(MonoArgs, CnArgs);
typedef void (*PipeFn)(MonoArgs, int);  // also the diffusion half of the split step
typedef std::vector<uint32_t> (*HaloFn)(bool);

struct ShapeEntry {
  int bi, bj, bk;
  StepFn iso, aniso;
  PipeFn pipe_iso, pipe_aniso;
  PipeFn diff_iso, diff_aniso;
  HaloFn halo;
  int stage_floats_iso, stage_floats_aniso;
  int diff_cap_iso, diff_cap_aniso;  // halo entries the diffusion kernel holds
  int diff_floats_iso, diff_floats_aniso;  // dynamic shared memory of the diffusion kernel
  CnFn cn_iso, cn_aniso;
  CnPassFn start_iso, start_aniso, apply_iso, apply_aniso;
};

#define HP_SHAPE(I, J, K)                                                                    \
  {I, J, K, mono_step_kernel<I, J, K, false>, mono_step_kernel<I, J, K, true>,               \
   mono_pipe_kernel<I, J, K, false>, mono_pipe_kernel<I, J, K, true>,                         \
   mono_diffuse_kernel<I, J, K, false>, mono_diffuse_kernel<I, J, K, true>, pipe_halo_table<I, J, K>, \
   PipeStage<I, J, K, false>::FLOATS, PipeStage<I, J, K, true>::FLOATS,                      \
   DiffHalo<I, J, K, false>::PER_THREAD * I * J * K, DiffHalo<I, J, K, true>::PER_THREAD * I * J * K, \
   DiffStage<I, J, K, false>::SMEM_FLOATS, DiffStage<I, J, K, true>::SMEM_FLOATS,            \
   cn_diag_kernel<I, J, K, false>, cn_diag_kernel<I, J, K, true>,                            \
   cn_pass_kernel<I, J, K, false, OP_CN_START>, cn_pass_kernel<I, J, K, true, OP_CN_START>,  \
   cn_pass_kernel<I, J, K, false, OP_CN_APPLY>, cn_pass_kernel<I, J, K, true, OP_CN_APPLY>}
static const ShapeEntry kShapes[] = {HP_SHAPE(4, 4, 8), HP_SHAPE(4, 8, 8), HP_SHAPE(2, 4, 16),
                                     HP_SHAPE(8, 8, 8)};
#undef HP_SHAPE

}  // namespace hp

using namespace hp;

struct HpMono {
  MonoArgs a;
  StepFn fn;
  PipeFn pipe;       // persistent pipelined step, or null
  int pipe_grid;     // CTAs of the persistent launch
  size_t pipe_smem;  // dynamic shared memory per CTA
  PipeFn diff;       // split step: diffusion half, or null
  int diff_grid;     // its persistent grid
  int ion_grid;      // grid of the ionic half
  size_t diff_smem;  // and dynamic shared memory per CTA
  CnFn cn;           // theta > 0: set-up pass (Jacobi diagonal), or null
  CnPassFn cn_start, cn_apply;  // tiled passes: start of a solve, A p
  CnArgs cn_a;
  int cn_grid;       // persistent grid of the set-up pass
  int cn_pgrid;      // persistent grid of the tiled passes
  int cn_vgrid;      // grid of the vector kernels
  int cn_chunk;      // iterations enqueued before the next flag test
  int32_t* cn_host;  // pinned copy of the done flag and iteration count
  cudaStream_t cn_body_stream;  // captures the bodies of the solve loops
  cudaGraphExec_t cn_graph;     // steps with device-side solve loops
  int cn_graph_steps;
  cudaStream_t cn_graph_stream;
  int bv;
  int64_t n_steps, steps_done;
  int64_t n_vm_frames, n_anim_frames;
  int anisotropic;
  std::vector<int32_t> slot_of_node;
  std::vector<void*> allocs;
  cudaGraphExec_t graph;
  int32_t graph_chunk;
  cudaStream_t graph_stream;
  int device;
};

template <typename T>
static hp_status up(HpMono* h, T** dst, const T* src, size_t n, cudaStream_t s) {
  hp_status st = dev_upload(dst, src, n, s);
  if (st == HP_OK && *dst) h->allocs.push_back((void*)*dst);
  return st;
}
template <typename T>
static hp_status al(HpMono* h, T** dst, size_t n) {
  hp_status st = dev_alloc(dst, n);
  if (st == HP_OK && *dst) h->allocs.push_back((void*)*dst);
  return st;
}

#define HP_TRY_NODESTROY(x)            \
  do {                                 \
    hp_status _s = (x);                \
    if (_s != HP_OK) return _s;        \
  } while (0)

#define HP_TRY(x)                      \
  do {                                 \
    hp_status _s = (x);                \
    if (_s != HP_OK) {                 \
      hp_mono_destroy(h);              \
      return _s;                       \
    }                                  \
  } while (0)

static hp_status launch_step(HpMono* h, int step_off, int mode, cudaStream_t s) {
  const int grid = h->a.n_bricks + (h->a.n_pk + h->bv - 1) / h->bv;
  if (grid == 0) return HP_OK;
  if (mode == 0 && h->diff) {
    h->diff<<<h->diff_grid, h->bv, h->diff_smem, s>>>(h->a, step_off);
    if (h->ion_grid > 0) mono_ionic_kernel<0><<<h->ion_grid, ION_THREADS, 0, s>>>(h->a, step_off);
  } else if (mode == 1 && h->diff) {
    if (h->ion_grid > 0) mono_ionic_kernel<1><<<h->ion_grid, ION_THREADS, 0, s>>>(h->a, step_off);
  } else if (mode == 0 && h->pipe)
    h->pipe<<<h->pipe_grid, h->bv, h->pipe_smem, s>>>(h->a, step_off);
  else
    h->fn<<<grid, h->bv, 0, s>>>(h->a, step_off, mode);
  HP_CUDA_TRY(cudaGetLastError());
  return HP_OK;
}

// Chooses the persistent pipelined step for a handle: uploads the shape's
// halo copy table, raises the dynamic shared-memory limit and sizes the grid
// to the resident CTAs of the whole GPU.  Without `required`, a shape whose
// two stages do not fit keeps the per-brick kernel.
static hp_status setup_pipe(HpMono* h, const ShapeEntry* se, int aniso, bool required,
                            cudaStream_t s) {
  const std::vector<uint32_t> tab = se->halo(aniso != 0);
  const int floats = aniso ? se->stage_floats_aniso : se->stage_floats_iso;
  const size_t smem = (2 * (size_t)floats + ((tab.size() + 3) & ~(size_t)3) + 54) * sizeof(float);
  const PipeFn fn = aniso ? se->pipe_aniso : se->pipe_iso;
  int dev = 0, max_optin = 0, n_sm = 0;
  HP_CUDA_TRY(cudaGetDevice(&dev));
  HP_CUDA_TRY(cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  HP_CUDA_TRY(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
  if (smem > (size_t)max_optin) {
    if (!required) return HP_OK;
    hp::set_error("hp_mono_create: pipelined kernel needs %zu B of shared memory, device has %d",
                  smem, max_optin);
    return HP_ERR_UNSUPPORTED;
  }
  HP_CUDA_TRY(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
  int per_sm = 0;
  HP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)fn, h->bv, smem));
  if (per_sm < 1) {
    if (!required) return HP_OK;
    hp::set_error("hp_mono_create: pipelined kernel cannot be resident");
    return HP_ERR_UNSUPPORTED;
  }
  uint32_t* dtab = nullptr;
  HP_TRY_NODESTROY(up(h, &dtab, tab.data(), tab.size(), s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));  // tab is a stack temporary
  h->a.halo_tab = dtab;
  h->a.n_halo = (int32_t)tab.size();
  const int n_items = h->a.n_bricks + (h->a.n_pk + h->bv - 1) / h->bv;
  h->pipe_grid = std::min(n_items, per_sm * n_sm);
  h->pipe_smem = smem;
  h->pipe = fn;
  return HP_OK;
}

// Split step: the compact list of tissue slots for the ionic launch.
static hp_status setup_split(HpMono* h, const ShapeEntry* se, const HpMonoDesc* d,
                             cudaStream_t s) {
  std::vector<int32_t> act;
  const int64_t ns = h->a.n_slots;
  act.reserve((size_t)ns);
  for (int64_t sl = 0; sl < ns; ++sl)
    if (d->tag[sl] & HP_TAG_PHENO_MASK) act.push_back((int32_t)sl);
  int32_t* dact = nullptr;
  HP_TRY_NODESTROY(up(h, &dact, act.data(), act.size(), s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));  // act is a stack temporary
  int shift = 0;
  while ((1 << shift) < h->bv) ++shift;
  h->a.active_slot = dact;
  h->a.n_active = (int32_t)act.size();
  h->a.n_active_pad = (int32_t)((act.size() + 31) / 32 * 32);
  h->a.bv_shift = shift;
  h->diff = d->anisotropic ? se->diff_aniso : se->diff_iso;
  // states in compact tissue order (resting state, as for the slot order)
  if (!act.empty())
    init_cells_kernel<<<1024, 256, 0, s>>>(h->a.state, h->a.Vpost, (int64_t)act.size(), d->v0);
  HP_CUDA_TRY(cudaGetLastError());
  // diffusion half: persistent CTAs over bricks, halo copy table per shape
  const std::vector<uint32_t> tab = se->halo(d->anisotropic != 0);
  if ((int)tab.size() > (d->anisotropic ? se->diff_cap_aniso : se->diff_cap_iso)) {
    hp::set_error("hp_mono_create: halo table of %zu entries exceeds the diffusion kernel's %d",
                  tab.size(), d->anisotropic ? se->diff_cap_aniso : se->diff_cap_iso);
    return HP_ERR_UNSUPPORTED;
  }
  uint32_t* dtab = nullptr;
  HP_TRY_NODESTROY(up(h, &dtab, tab.data(), tab.size(), s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));  // tab is a stack temporary
  h->a.halo_tab = dtab;
  h->a.n_halo = (int32_t)tab.size();
  const size_t smem =
      (size_t)(d->anisotropic ? se->diff_floats_aniso : se->diff_floats_iso) * sizeof(float);
  int dev = 0, n_sm = 0, per_sm = 0;
  HP_CUDA_TRY(cudaGetDevice(&dev));
  HP_CUDA_TRY(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
  HP_CUDA_TRY(cudaFuncSetAttribute((const void*)h->diff, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
  HP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)h->diff, h->bv, smem));
  h->diff_smem = smem;
  const int n_items = h->a.n_bricks + (h->a.n_pk + h->bv - 1) / h->bv;
  h->diff_grid = std::max(1, std::min(n_items, std::max(per_sm, 1) * n_sm));
  h->ion_grid = (h->a.n_active_pad + h->a.n_pk + ION_THREADS - 1) / ION_THREADS;
  return HP_OK;
}

// Theta-scheme diffusion half: CG vectors, the grids of the tiled passes and
// the vector kernels, and the Jacobi diagonal (cn_diag_kernel, once).
static hp_status setup_cn(HpMono* h, const ShapeEntry* se, const HpMonoDesc* d, cudaStream_t s) {
  CnArgs& c = h->cn_a;
  memset(&c, 0, sizeof(c));
  const int64_t n = h->a.n_slots + h->a.n_pk;
  c.n = n;
  c.theta = (float)d->theta;
  c.omt = (float)(1.0 - d->theta);
  c.pk_weight = d->pk_weight;
  // the vectors are FP32: a tighter relative tolerance than ~1e-7 is not
  // reachable by the recursive residual
  const double tol = std::max(d->cn_tol, 1e-7);
  c.tol2 = tol * tol;
  c.max_iter = d->cn_max_iter;
  h->cn = d->anisotropic ? se->cn_aniso : se->cn_iso;
  h->cn_start = d->anisotropic ? se->start_aniso : se->start_iso;
  h->cn_apply = d->anisotropic ? se->apply_aniso : se->apply_iso;
  int dev = 0, n_sm = 0, per_sm = 0, per_sm_s = 0, per_sm_a = 0;
  HP_CUDA_TRY(cudaGetDevice(&dev));
  HP_CUDA_TRY(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
  HP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)h->cn, h->bv, 0));
  const int n_items = h->a.n_bricks + (h->a.n_pk + h->bv - 1) / h->bv;
  h->cn_grid = std::max(1, std::min(n_items, std::max(per_sm, 1) * n_sm));
  // the tiled passes use the split diffusion kernel's shared-memory stages
  for (CnPassFn f : {h->cn_start, h->cn_apply})
    HP_CUDA_TRY(cudaFuncSetAttribute((const void*)f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)h->diff_smem));
  HP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_s, (const void*)h->cn_start,
                                                            h->bv, h->diff_smem));
  HP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_a, (const void*)h->cn_apply,
                                                            h->bv, h->diff_smem));
  h->cn_pgrid = std::max(1, std::min(n_items, std::max(std::min(per_sm_s, per_sm_a), 1) * n_sm));
  h->cn_vgrid = (int)std::max<int64_t>(1, std::min<int64_t>((n + CN_TB - 1) / CN_TB, 8 * n_sm));
  h->cn_chunk = 4;
  HP_TRY_NODESTROY(al(h, &c.x, n));
  HP_TRY_NODESTROY(al(h, &c.r, n));
  HP_TRY_NODESTROY(al(h, &c.p, n));
  HP_TRY_NODESTROY(al(h, &c.q, n));
  HP_TRY_NODESTROY(al(h, &c.dinv, n));
  HP_TRY_NODESTROY(al(h, &c.part,
                       (size_t)std::max({h->cn_grid, h->cn_pgrid, h->cn_vgrid}) * CN_NPART));
  HP_TRY_NODESTROY(al(h, &c.scal, N_CN_SCAL));
  HP_TRY_NODESTROY(al(h, &c.iscal, N_CN_ISCAL));
  HP_TRY_NODESTROY(al(h, &c.ticket, 1));
  HP_CUDA_TRY(cudaMemsetAsync(c.scal, 0, N_CN_SCAL * sizeof(double), s));
  HP_CUDA_TRY(cudaMemsetAsync(c.iscal, 0, N_CN_ISCAL * sizeof(int32_t), s));
  HP_CUDA_TRY(cudaMemsetAsync(c.ticket, 0, sizeof(unsigned int), s));
  // padding entries of the CG vectors stay zero (the passes skip them)
  for (float* v : {c.x, c.r, c.p, c.q}) HP_CUDA_TRY(cudaMemsetAsync(v, 0, n * sizeof(float), s));
  HP_CUDA_TRY(cudaMallocHost((void**)&h->cn_host, 2 * sizeof(int32_t)));
  h->a.cn_x = c.x;
  HP_CUDA_TRY(cudaStreamCreateWithFlags(&h->cn_body_stream, cudaStreamNonBlocking));
  h->cn<<<h->cn_grid, h->bv, 0, s>>>(h->a, c);
  HP_CUDA_TRY(cudaGetLastError());
  return HP_OK;
}

// One CG iteration of the theta-scheme solve: q = M p (tiled pass, alpha),
// x and r updates (beta, stopping test), new direction.  Every kernel
// returns at once once the done flag is set.
static void cn_iteration(HpMono* h, cudaStream_t s) {
  const CnArgs& c = h->cn_a;
  h->cn_apply<<<h->cn_pgrid, h->bv, h->diff_smem, s>>>(h->a, c);
  cn_update_kernel<<<h->cn_vgrid, CN_TB, 0, s>>>(c, h->a.n_slots);
  cn_dir_kernel<<<h->cn_vgrid, CN_TB, 0, s>>>(c);
}

// One theta-scheme step: the stencil pass that starts the solve, CG
// iterations in chunks (sized by the previous step's count) until the done
// flag, the outputs of V_{i+1} = clamp(x) with the ionic half (one launch)
// and the step count.
static hp_status cn_step(HpMono* h, cudaStream_t s) {
  const CnArgs& c = h->cn_a;
  h->cn_start<<<h->cn_pgrid, h->bv, h->diff_smem, s>>>(h->a, c);
  HP_CUDA_TRY(cudaGetLastError());
  int launched = 0;
  while (launched < c.max_iter) {
    const int k = std::min(h->cn_chunk, c.max_iter - launched);
    for (int j = 0; j < k; ++j) cn_iteration(h, s);
    HP_CUDA_TRY(cudaGetLastError());
    launched += k;
    HP_CUDA_TRY(cudaMemcpyAsync(h->cn_host, c.iscal + CI_DONE, 2 * sizeof(int32_t),
                                cudaMemcpyDeviceToHost, s));
    HP_CUDA_TRY(cudaStreamSynchronize(s));
    if (h->cn_host[0]) break;
  }
  // next step: enqueue this step's count (+1) before the first test
  h->cn_chunk = std::max(1, std::min(h->cn_host[1] + 1, 64));
  if (h->ion_grid > 0) mono_ionic_kernel<2><<<h->ion_grid, ION_THREADS, 0, s>>>(h->a, 0);
  advance_kernel<<<1, 1, 0, s>>>((int64_t*)h->a.d_step, 1);
  HP_CUDA_TRY(cudaGetLastError());
  return HP_OK;
}

// Captures n theta-scheme steps on s (which is capturing): per step the
// start pass, the loop-condition kernel and a conditional WHILE node whose
// body (captured on cn_body_stream) is one CG iteration plus the condition
// update, then the outputs, the ionic half and the step count.  No host
// round trip per step.
static hp_status cn_capture_steps(HpMono* h, int n, cudaStream_t s) {
  const CnArgs& c = h->cn_a;
  cudaStream_t sb = h->cn_body_stream;
  for (int k = 0; k < n; ++k) {
    h->cn_start<<<h->cn_pgrid, h->bv, h->diff_smem, s>>>(h->a, c);
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    HP_CUDA_TRY(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
    cudaGraphConditionalHandle hd;
    HP_CUDA_TRY(cudaGraphConditionalHandleCreate(&hd, g, 0, 0));
    cn_cond_kernel<<<1, 1, 0, s>>>(hd, c, 1);
    HP_CUDA_TRY(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
    cudaGraphNodeParams np = {cudaGraphNodeTypeConditional};
    np.conditional.handle = hd;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    HP_CUDA_TRY(cudaGraphAddNode(&node, g, deps, nd, &np));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    HP_CUDA_TRY(cudaStreamBeginCaptureToGraph(sb, body, nullptr, nullptr, 0,
                                              cudaStreamCaptureModeRelaxed));
    cn_iteration(h, sb);
    cn_cond_kernel<<<1, 1, 0, sb>>>(hd, c, 0);
    cudaGraph_t bo = nullptr;
    HP_CUDA_TRY(cudaStreamEndCapture(sb, &bo));
    HP_CUDA_TRY(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    if (h->ion_grid > 0) mono_ionic_kernel<2><<<h->ion_grid, ION_THREADS, 0, s>>>(h->a, 0);
    advance_kernel<<<1, 1, 0, s>>>((int64_t*)h->a.d_step, 1);
    HP_CUDA_TRY(cudaGetLastError());
  }
  return HP_OK;
}

// (Re)builds the graph of n theta-scheme steps for stream s.
static hp_status cn_build_graph(HpMono* h, int n, cudaStream_t s) {
  if (h->cn_graph) {
    cudaGraphExecDestroy(h->cn_graph);
    h->cn_graph = nullptr;
  }
  HP_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  const hp_status st = cn_capture_steps(h, n, s);
  cudaStreamCaptureStatus bs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(h->cn_body_stream, &bs) == cudaSuccess &&
      bs != cudaStreamCaptureStatusNone) {
    cudaGraph_t dead = nullptr;
    cudaStreamEndCapture(h->cn_body_stream, &dead);
  }
  cudaGraph_t g = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(s, &g);
  if (st != HP_OK) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  HP_CUDA_TRY(ce);
  const cudaError_t ie = cudaGraphInstantiate(&h->cn_graph, g, 0);
  cudaGraphDestroy(g);
  HP_CUDA_TRY(ie);
  h->cn_graph_steps = n;
  h->cn_graph_stream = s;
  return HP_OK;
}

extern "C" hp_status hp_mono_create(const HpMonoDesc* d, HpMono** out, void* stream) {
  HP_REQUIRE(d && out, "hp_mono_create: null argument");
  *out = nullptr;
  const ShapeEntry* se = nullptr;
  for (const auto& e : kShapes)
    if (e.bi == d->bi && e.bj == d->bj && e.bk == d->bk) se = &e;
  if (!se) {
    hp::set_error("hp_mono_create: brick shape %dx%dx%d is not compiled", d->bi, d->bj, d->bk);
    return HP_ERR_UNSUPPORTED;
  }
  HP_REQUIRE(d->n_bricks >= 0 && d->n_pk >= 0, "hp_mono_create: negative sizes");
  HP_REQUIRE(d->n_sites >= 0 && d->n_sites <= HP_MAX_SITES, "hp_mono_create: n_sites must be 0..%d",
             HP_MAX_SITES);
  HP_REQUIRE(d->n_variants >= 1 && d->n_variants <= HP_MAX_VARIANTS,
             "hp_mono_create: n_variants must be 1..%d", HP_MAX_VARIANTS);
  HP_REQUIRE(d->max_events >= 1 && d->max_events <= 16, "hp_mono_create: max_events must be 1..16");
  HP_REQUIRE(d->dt > 0.0 && d->Cm > 0.0, "hp_mono_create: dt and Cm must be positive");
  HP_REQUIRE(d->n_steps >= 0, "hp_mono_create: n_steps must be >= 0");
  HP_REQUIRE(d->n_bricks == 0 || (d->brick_nbr && d->tag), "hp_mono_create: missing brick arrays");
  HP_REQUIRE(!d->anisotropic || d->n_bricks == 0 || (d->wface && d->doff),
             "hp_mono_create: anisotropic needs wface and doff");
  HP_REQUIRE(d->n_pk == 0 || (d->pk_ptr && d->pk_stim), "hp_mono_create: missing Purkinje arrays");
  HP_REQUIRE(d->site_on && (d->n_sites == 0 || d->site_amp), "hp_mono_create: missing site tables");
  HP_REQUIRE(d->n_myo >= 0 && (d->n_myo == 0 || d->slot_of_node), "hp_mono_create: missing slot_of_node");
  HP_REQUIRE(d->kernel >= 0 && d->kernel <= 3, "hp_mono_create: kernel must be 0..3");
  HP_REQUIRE(d->theta >= 0.0 && d->theta <= 1.0, "hp_mono_create: theta must be in [0, 1]");
  HP_REQUIRE(d->theta == 0.0 ||
                 (d->cn_tol > 0.0 && d->cn_max_iter >= 1 && (d->n_pk == 0 || d->pk_weight > 0.0f)),
             "hp_mono_create: theta > 0 needs cn_tol > 0, cn_max_iter >= 1 and pk_weight > 0");
  HP_REQUIRE(d->theta == 0.0 || d->kernel == HP_MONO_KERNEL_AUTO || d->kernel == HP_MONO_KERNEL_SPLIT,
             "hp_mono_create: theta > 0 runs on the split step (kernel AUTO or SPLIT)");

  HpMono* h = new HpMono();
  h->graph = nullptr;
  h->graph_chunk = 0;
  h->graph_stream = nullptr;
  cudaGetDevice(&h->device);
  cudaStream_t s = (cudaStream_t)stream;
  MonoArgs& a = h->a;
  memset(&a, 0, sizeof(a));
  h->bv = d->bi * d->bj * d->bk;
  h->fn = d->anisotropic ? se->aniso : se->iso;
  h->pipe = nullptr;
  h->pipe_grid = 0;
  h->pipe_smem = 0;
  h->diff = nullptr;
  h->diff_grid = 0;
  h->diff_smem = 0;
  h->ion_grid = 0;
  h->cn = nullptr;
  h->cn_host = nullptr;
  h->cn_body_stream = nullptr;
  h->cn_graph = nullptr;
  h->cn_graph_steps = 0;
  h->cn_graph_stream = nullptr;
  h->anisotropic = d->anisotropic;
  h->n_steps = d->n_steps;
  h->steps_done = 0;
  a.n_bricks = d->n_bricks;
  a.n_pk = d->n_pk;
  const int64_t ns = (int64_t)d->n_bricks * h->bv;
  a.n_slots = ns;
  HP_TRY(up(h, (uint32_t**)&a.tag, d->tag, ns, s));
  if (d->anisotropic) {
    HP_TRY(up(h, (float**)&a.wface, d->wface, 3 * ns, s));
    HP_TRY(up(h, (float**)&a.doff, d->doff, 3 * ns, s));
  }
  a.iso_coef = d->iso_coef;
  HP_TRY(up(h, (int32_t**)&a.nbr, d->brick_nbr, (size_t)27 * d->n_bricks, s));
  if (d->brick_variant) HP_TRY(up(h, (uint8_t**)&a.brick_variant, d->brick_variant, d->n_bricks, s));
  HP_TRY(al(h, &a.state, (size_t)N_STATE * ns));
  HP_TRY(al(h, &a.Vs0, ns));
  HP_TRY(al(h, &a.Vs1, ns));
  HP_TRY(al(h, &a.Vpost, ns));
  // Purkinje
  if (d->n_pk > 0) {
    HP_TRY(up(h, (int32_t**)&a.pk_ptr, d->pk_ptr, d->n_pk + 1, s));
    const int32_t nnz = d->pk_ptr[d->n_pk];
    HP_REQUIRE(nnz >= 0, "hp_mono_create: bad pk_ptr");
    if (nnz > 0) {
      HP_REQUIRE(d->pk_idx && d->pk_coef, "hp_mono_create: missing pk_idx/pk_coef");
      for (int32_t q = 0; q < nnz; ++q) {
        const int32_t j = d->pk_idx[q];
        if (j >= d->n_pk || (j < 0 && -(int64_t)j - 1 >= ns)) {
          hp::set_error("hp_mono_create: pk_idx[%d]=%d out of range", q, j);
          hp_mono_destroy(h);
          return HP_ERR_INVALID;
        }
      }
      HP_TRY(up(h, (int32_t**)&a.pk_idx, d->pk_idx, nnz, s));
      HP_TRY(up(h, (float**)&a.pk_coef, d->pk_coef, nnz, s));
    }
    HP_TRY(up(h, (uint8_t**)&a.pk_stim, d->pk_stim, d->n_pk, s));
    if (d->pk_variant) HP_TRY(up(h, (uint8_t**)&a.pk_variant, d->pk_variant, d->n_pk, s));
    HP_TRY(al(h, &a.pk_state, (size_t)N_STATE * d->n_pk));
    HP_TRY(al(h, &a.pk_Vs0, d->n_pk));
    HP_TRY(al(h, &a.pk_Vs1, d->n_pk));
    HP_TRY(al(h, &a.pk_Vpost, d->n_pk));
  }
  if (d->n_pmj_rows > 0) {
    HP_REQUIRE(d->pmj_row && d->pmj_ptr, "hp_mono_create: missing junction arrays");
    const int32_t nnz = d->pmj_ptr[d->n_pmj_rows];
    for (int32_t q = 0; q < nnz; ++q)
      if (d->pmj_pk[q] < 0 || d->pmj_pk[q] >= d->n_pk) {
        hp::set_error("hp_mono_create: pmj_pk[%d] out of range", q);
        hp_mono_destroy(h);
        return HP_ERR_INVALID;
      }
    HP_TRY(up(h, (int32_t**)&a.pmj_row, d->pmj_row, ns, s));
    HP_TRY(up(h, (int32_t**)&a.pmj_ptr, d->pmj_ptr, d->n_pmj_rows + 1, s));
    HP_TRY(up(h, (int32_t**)&a.pmj_pk, d->pmj_pk, nnz, s));
    HP_TRY(up(h, (float**)&a.pmj_coef, d->pmj_coef, nnz, s));
  }
  // time stepping
  a.dt_d = d->dt;
  a.dt = (float)d->dt;
  a.Cm = (float)d->Cm;
  a.dt_over_Cm = (float)(d->dt / d->Cm);
  {
    // per-variant site tables: amplitudes padded to HP_MAX_SITES per variant
    std::vector<float> amp((size_t)d->n_variants * HP_MAX_SITES, 0.0f);
    for (int v = 0; v < d->n_variants; ++v)
      for (int i = 0; i < d->n_sites; ++i)
        amp[(size_t)v * HP_MAX_SITES + i] = d->site_amp[(size_t)v * d->n_sites + i];
    HP_TRY(up(h, (float**)&a.site_amp, amp.data(), amp.size(), s));
    HP_CUDA_TRY(cudaStreamSynchronize(s));  // amp is a stack temporary
  }
  a.site_stride = d->n_steps + 1;
  HP_TRY(up(h, (uint8_t**)&a.site_on, d->site_on, (size_t)d->n_variants * (d->n_steps + 1), s));
  HP_TRY(up(h, (float**)&a.var_gks, d->variant_gks, d->n_variants, s));
  HP_TRY(up(h, (float**)&a.var_gkr, d->variant_gkr, d->n_variants, s));
  // outputs
  a.n_myo = d->n_myo;
  h->slot_of_node.assign(d->slot_of_node, d->slot_of_node + d->n_myo);
  {
    std::vector<int32_t> node_of_slot(ns, -1);
    for (int32_t i = 0; i < d->n_myo; ++i) {
      const int32_t sl = d->slot_of_node[i];
      if (sl < 0 || sl >= ns) {
        hp::set_error("hp_mono_create: slot_of_node[%d]=%d out of range", i, sl);
        hp_mono_destroy(h);
        return HP_ERR_INVALID;
      }
      node_of_slot[sl] = i;
    }
    // every tissue slot must map to a node (snapshots scatter through it)
    for (int64_t sl = 0; sl < ns; ++sl)
      if ((d->tag[sl] & HP_TAG_PHENO_MASK) && node_of_slot[sl] < 0) {
        hp::set_error("hp_mono_create: tissue slot %lld has no node", (long long)sl);
        hp_mono_destroy(h);
        return HP_ERR_INVALID;
      }
    HP_TRY(up(h, (int32_t**)&a.node_of_slot, node_of_slot.data(), ns, s));
    HP_CUDA_TRY(cudaStreamSynchronize(s));  // node_of_slot is a stack temporary
  }
  a.vm_every = d->vm_every;
  h->n_vm_frames = d->vm_every > 0 ? (d->n_steps + d->vm_every - 1) / d->vm_every : 0;
  HP_TRY(al(h, &a.vm_snap, (size_t)h->n_vm_frames * d->n_myo));
  a.frame_every = d->frame_every;
  h->n_anim_frames = d->frame_every > 0 ? (d->n_steps + d->frame_every - 1) / d->frame_every : 0;
  a.n_surf = d->n_surf;
  if (d->n_surf > 0) {
    HP_REQUIRE(d->surf_of_slot, "hp_mono_create: missing surf_of_slot");
    HP_TRY(up(h, (int32_t**)&a.surf_of_slot, d->surf_of_slot, ns, s));
  }
  HP_TRY(al(h, &a.surf_frames, (size_t)h->n_anim_frames * d->n_surf));
  HP_TRY(al(h, &a.pk_frames, (size_t)h->n_anim_frames * d->n_pk));
  a.act_thr = d->act_threshold;
  a.deact_thr = d->deact_threshold;
  a.max_events = d->max_events;
  HP_TRY(al(h, &a.act_t, (size_t)d->max_events * ns));
  HP_TRY(al(h, &a.deact_t, (size_t)d->max_events * ns));
  HP_TRY(al(h, &a.act_n, ns));
  HP_TRY(al(h, &a.deact_n, ns));
  if (ns) {
    HP_CUDA_TRY(cudaMemsetAsync(a.act_n, 0, ns, s));
    HP_CUDA_TRY(cudaMemsetAsync(a.deact_n, 0, ns, s));
    HP_CUDA_TRY(cudaMemsetAsync(a.Vs1, 0, ns * sizeof(float), s));
  }
  int64_t* dstep = nullptr;
  HP_TRY(al(h, &dstep, 1));
  HP_CUDA_TRY(cudaMemsetAsync(dstep, 0, sizeof(int64_t), s));
  a.d_step = dstep;
  const float nanv = nanf("");
  if (ns) {
    fill_kernel<<<1024, 256, 0, s>>>(a.act_t, (int64_t)d->max_events * ns, nanv);
    fill_kernel<<<1024, 256, 0, s>>>(a.deact_t, (int64_t)d->max_events * ns, nanv);
    init_cells_kernel<<<1024, 256, 0, s>>>(a.state, a.Vpost, ns, d->v0);
  }
  if (d->n_pk) {
    init_cells_kernel<<<256, 256, 0, s>>>(a.pk_state, a.pk_Vpost, d->n_pk, d->v0);
    HP_CUDA_TRY(cudaMemsetAsync(a.pk_Vs1, 0, d->n_pk * sizeof(float), s));
  }
  HP_CUDA_TRY(cudaGetLastError());
  if (d->kernel == HP_MONO_KERNEL_SPLIT || d->theta > 0.0 ||
      (d->kernel == HP_MONO_KERNEL_AUTO && d->n_bricks > 0)) {
    HP_TRY(setup_split(h, se, d, s));
    if (d->theta > 0.0) HP_TRY(setup_cn(h, se, d, s));
  } else if (d->kernel != HP_MONO_KERNEL_BRICK && d->n_bricks > 0) {
    HP_TRY(setup_pipe(h, se, d->anisotropic, d->kernel == HP_MONO_KERNEL_PIPELINED, s));
  }
  HP_TRY(launch_step(h, 0, 1, s));  // W_0 = ionic(V_0)
  // the caller's host arrays may be released once this returns
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  *out = h;
  return HP_OK;
}

extern "C" hp_status hp_mono_run(HpMono* h, int64_t n, int32_t graph_chunk, void* stream) {
  HP_REQUIRE(h, "hp_mono_run: null handle");
  HP_REQUIRE(n >= 0 && h->steps_done + n <= h->n_steps,
             "hp_mono_run: %lld steps requested, %lld remain", (long long)n,
             (long long)(h->n_steps - h->steps_done));
  cudaStream_t s = (cudaStream_t)stream;
  if (h->cn) {
    // theta-scheme: graphs of up to 16 steps whose solve loops run on the
    // device (conditional nodes); the remainder, and the legacy default
    // stream that cannot be captured, test convergence on the host
    int64_t left = n;
    const int gs = (int)std::min<int64_t>(graph_chunk, 16);
    if (gs > 0 && left >= gs && s != nullptr) {
      if (!h->cn_graph || h->cn_graph_steps != gs || h->cn_graph_stream != s)
        HP_TRY_NODESTROY(cn_build_graph(h, gs, s));
      while (left >= gs) {
        HP_CUDA_TRY(cudaGraphLaunch(h->cn_graph, s));
        left -= gs;
        h->steps_done += gs;
      }
    }
    for (; left > 0; --left) {
      hp_status st = cn_step(h, s);
      if (st != HP_OK) return st;
      h->steps_done += 1;
    }
    return HP_OK;
  }
  int64_t left = n;
  // the legacy default stream cannot be captured: launch directly there
  if (graph_chunk > 0 && left >= graph_chunk && s != nullptr) {
    if (!h->graph || h->graph_chunk != graph_chunk || h->graph_stream != s) {
      if (h->graph) {
        cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
      }
      cudaGraph_t g;
      HP_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      hp_status st = HP_OK;
      for (int o = 0; o < graph_chunk && st == HP_OK; ++o) st = launch_step(h, o, 0, s);
      if (st == HP_OK) advance_kernel<<<1, 1, 0, s>>>((int64_t*)h->a.d_step, graph_chunk);
      cudaError_t ce = cudaStreamEndCapture(s, &g);
      if (st != HP_OK) return st;
      HP_CUDA_TRY(ce);
      HP_CUDA_TRY(cudaGraphInstantiate(&h->graph, g, 0));
      cudaGraphDestroy(g);
      h->graph_chunk = graph_chunk;
      h->graph_stream = s;
    }
    while (left >= graph_chunk) {
      HP_CUDA_TRY(cudaGraphLaunch(h->graph, s));
      left -= graph_chunk;
    }
  }
  if (left > 0) {
    for (int64_t o = 0; o < left; ++o) {
      hp_status st = launch_step(h, (int)o, 0, s);
      if (st != HP_OK) return st;
    }
    advance_kernel<<<1, 1, 0, s>>>((int64_t*)h->a.d_step, left);
    HP_CUDA_TRY(cudaGetLastError());
  }
  h->steps_done += n;
  return HP_OK;
}

extern "C" int64_t hp_mono_steps_done(const HpMono* h) { return h ? h->steps_done : -1; }

extern "C" hp_status hp_mono_kernel_info(const HpMono* h, int32_t* kernel, int32_t* grid,
                                         int64_t* smem_bytes) {
  HP_REQUIRE(h, "hp_mono_kernel_info: null handle");
  if (kernel)
    *kernel = h->diff ? HP_MONO_KERNEL_SPLIT
                      : (h->pipe ? HP_MONO_KERNEL_PIPELINED : HP_MONO_KERNEL_BRICK);
  if (grid)
    *grid = h->diff ? h->diff_grid
                    : (h->pipe ? h->pipe_grid : h->a.n_bricks + (h->a.n_pk + h->bv - 1) / h->bv);
  if (smem_bytes) *smem_bytes = h->pipe ? (int64_t)h->pipe_smem : 0;
  return HP_OK;
}

extern "C" hp_status hp_mono_copy_vm(HpMono* h, int64_t f0, int64_t nf, float* dst,
                                     int32_t dst_on_device, void* stream) {
  HP_REQUIRE(h && dst, "hp_mono_copy_vm: null argument");
  HP_REQUIRE(f0 >= 0 && nf >= 0 && f0 + nf <= h->n_vm_frames,
             "hp_mono_copy_vm: frames [%lld,%lld) outside [0,%lld)", (long long)f0,
             (long long)(f0 + nf), (long long)h->n_vm_frames);
  if (nf == 0 || h->a.n_myo == 0) return HP_OK;
  HP_CUDA_TRY(cudaMemcpyAsync(dst, h->a.vm_snap + f0 * h->a.n_myo, nf * h->a.n_myo * sizeof(float),
                              dst_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                              (cudaStream_t)stream));
  return HP_OK;
}

extern "C" hp_status hp_mono_copy_frames(HpMono* h, int64_t f0, int64_t nf, float* dst_surf,
                                         float* dst_pk, int32_t dst_on_device, void* stream) {
  HP_REQUIRE(h, "hp_mono_copy_frames: null handle");
  HP_REQUIRE(f0 >= 0 && nf >= 0 && f0 + nf <= h->n_anim_frames,
             "hp_mono_copy_frames: frames out of range");
  const cudaMemcpyKind k = dst_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  cudaStream_t s = (cudaStream_t)stream;
  if (dst_surf && h->a.n_surf && nf)
    HP_CUDA_TRY(cudaMemcpyAsync(dst_surf, h->a.surf_frames + f0 * h->a.n_surf,
                                nf * h->a.n_surf * sizeof(float), k, s));
  if (dst_pk && h->a.n_pk && nf)
    HP_CUDA_TRY(cudaMemcpyAsync(dst_pk, h->a.pk_frames + f0 * h->a.n_pk,
                                nf * h->a.n_pk * sizeof(float), k, s));
  return HP_OK;
}

extern "C" hp_status hp_mono_copy_events(HpMono* h, float* act, int32_t* n_act, float* deact,
                                         int32_t* n_deact, void* stream) {
  HP_REQUIRE(h, "hp_mono_copy_events: null handle");
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t ns = h->a.n_slots, nm = h->a.n_myo;
  const int me = h->a.max_events;
  std::vector<float> t((size_t)me * ns);
  std::vector<uint8_t> c(ns);
  for (int pass = 0; pass < 2; ++pass) {
    float* dt_ = pass ? deact : act;
    int32_t* dn = pass ? n_deact : n_act;
    if (!dt_ && !dn) continue;
    if (ns) {
      HP_CUDA_TRY(cudaMemcpyAsync(t.data(), pass ? h->a.deact_t : h->a.act_t,
                                  t.size() * sizeof(float), cudaMemcpyDeviceToHost, s));
      HP_CUDA_TRY(cudaMemcpyAsync(c.data(), pass ? h->a.deact_n : h->a.act_n, ns,
                                  cudaMemcpyDeviceToHost, s));
      HP_CUDA_TRY(cudaStreamSynchronize(s));
    }
    for (int64_t i = 0; i < nm; ++i) {
      const int32_t sl = h->slot_of_node[i];
      if (dn) dn[i] = c[sl];
      if (dt_)
        for (int e = 0; e < me; ++e) dt_[(int64_t)e * nm + i] = t[(size_t)e * ns + sl];
    }
  }
  return HP_OK;
}

namespace hp {
__global__ void w_gather_kernel(const float* __restrict__ W, const int32_t* __restrict__ slots,
                                int64_t n, float* __restrict__ out) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x)
    out[q] = W[slots[q]];
}
__global__ void w_scatter_kernel(float* __restrict__ W, const int32_t* __restrict__ slots,
                                 int64_t n, const float* __restrict__ in) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x)
    W[slots[q]] = in[q];
}
}  // namespace hp

// The W buffer the next step's diffusion half reads (step steps_done).
static float* next_w(HpMono* h) { return (h->steps_done & 1) ? h->a.Vs1 : h->a.Vs0; }

extern "C" hp_status hp_mono_w_gather(HpMono* h, const int32_t* slots, int64_t n, float* out,
                                      void* stream) {
  HP_REQUIRE(h && (n == 0 || (slots && out)), "hp_mono_w_gather: null argument");
  HP_REQUIRE(n >= 0, "hp_mono_w_gather: negative count");
  HP_REQUIRE(!h->cn, "hp_mono_w_gather: the slab exchange runs the explicit step (theta = 0)");
  if (n == 0) return HP_OK;
  const int grid = (int)std::min<int64_t>((n + 255) / 256, 4096);
  w_gather_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(next_w(h), slots, n, out);
  HP_CUDA_TRY(cudaGetLastError());
  return HP_OK;
}

extern "C" hp_status hp_mono_w_scatter(HpMono* h, const int32_t* slots, int64_t n,
                                       const float* in, void* stream) {
  HP_REQUIRE(h && (n == 0 || (slots && in)), "hp_mono_w_scatter: null argument");
  HP_REQUIRE(n >= 0, "hp_mono_w_scatter: negative count");
  HP_REQUIRE(!h->cn, "hp_mono_w_scatter: the slab exchange runs the explicit step (theta = 0)");
  if (n == 0) return HP_OK;
  const int grid = (int)std::min<int64_t>((n + 255) / 256, 4096);
  w_scatter_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(next_w(h), slots, n, in);
  HP_CUDA_TRY(cudaGetLastError());
  return HP_OK;
}

extern "C" hp_status hp_mono_copy_v(HpMono* h, float* v_myo, float* v_pk, void* stream) {
  HP_REQUIRE(h, "hp_mono_copy_v: null handle");
  cudaStream_t s = (cudaStream_t)stream;
  if (v_myo && h->a.n_myo) {
    std::vector<float> v(h->a.n_slots);
    HP_CUDA_TRY(cudaMemcpyAsync(v.data(), h->a.Vpost, v.size() * sizeof(float),
                                cudaMemcpyDeviceToHost, s));
    HP_CUDA_TRY(cudaStreamSynchronize(s));
    for (int64_t i = 0; i < h->a.n_myo; ++i) v_myo[i] = v[h->slot_of_node[i]];
  }
  if (v_pk && h->a.n_pk) {
    HP_CUDA_TRY(cudaMemcpyAsync(v_pk, h->a.pk_Vpost, h->a.n_pk * sizeof(float),
                                cudaMemcpyDeviceToHost, s));
    HP_CUDA_TRY(cudaStreamSynchronize(s));
  }
  return HP_OK;
}

extern "C" hp_status hp_mono_copy_state(HpMono* h, float* st_slots, float* st_pk, void* stream) {
  HP_REQUIRE(h, "hp_mono_copy_state: null handle");
  cudaStream_t s = (cudaStream_t)stream;
  if (st_slots && h->a.n_slots) {
    HP_CUDA_TRY(cudaMemcpyAsync(st_slots, h->a.state, (size_t)N_STATE * h->a.n_slots * sizeof(float),
                                cudaMemcpyDeviceToHost, s));
    if (h->diff) {
      // the split step stores states in compact tissue order: scatter to slots
      HP_CUDA_TRY(cudaStreamSynchronize(s));
      const int64_t ns = h->a.n_slots, na = h->a.n_active;
      std::vector<int32_t> act(na);
      if (na) HP_CUDA_TRY(cudaMemcpy(act.data(), h->a.active_slot, na * 4, cudaMemcpyDeviceToHost));
      std::vector<float> tmp((size_t)N_STATE * na);
      for (int v = 0; v < N_STATE; ++v)
        std::copy(st_slots + (size_t)v * na, st_slots + (size_t)(v + 1) * na, tmp.begin() + (size_t)v * na);
      for (int v = 0; v < N_STATE; ++v) {
        float* dst = st_slots + (size_t)v * ns;
        std::fill(dst, dst + ns, 0.0f);
        for (int64_t i = 0; i < na; ++i) dst[act[i]] = tmp[(size_t)v * na + i];
      }
    }
  }
  if (st_pk && h->a.n_pk)
    HP_CUDA_TRY(cudaMemcpyAsync(st_pk, h->a.pk_state, (size_t)N_STATE * h->a.n_pk * sizeof(float),
                                cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  return HP_OK;
}

extern "C" hp_status hp_mono_cn_stats(HpMono* h, int64_t* iterations, int64_t* solves,
                                      int64_t* unconverged, int64_t* breakdowns) {
  HP_REQUIRE(h, "hp_mono_cn_stats: null handle");
  int32_t v[N_CN_ISCAL] = {0};
  if (h->cn) HP_CUDA_TRY(cudaMemcpy(v, h->cn_a.iscal, sizeof(v), cudaMemcpyDeviceToHost));
  if (iterations) *iterations = v[CI_TOTAL];
  if (solves) *solves = v[CI_SOLVES];
  if (unconverged) *unconverged = v[CI_UNCONV];
  if (breakdowns) *breakdowns = v[CI_BREAK];
  return HP_OK;
}

extern "C" hp_status hp_mono_destroy(HpMono* h) {
  if (!h) return HP_OK;
  if (h->graph) cudaGraphExecDestroy(h->graph);
  if (h->cn_graph) cudaGraphExecDestroy(h->cn_graph);
  if (h->cn_body_stream) cudaStreamDestroy(h->cn_body_stream);
  if (h->cn_host) cudaFreeHost(h->cn_host);
  for (void* p : h->allocs) cudaFree(p);
  delete h;
  return HP_OK;
}
