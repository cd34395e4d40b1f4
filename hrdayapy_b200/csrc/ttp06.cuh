// TTP06 (ten Tusscher & Panfilov 2006) single-cell update in FP32.  Same
// kinetics as HrdayaPy's
// simulation/functions/ionic_models/gpu_ttp06.py:198-412 (_currents_and_gates):
// Rush-Larsen for the 12 gates, forward Euler for Rprime and the five
// concentrations with the reference's clamps, phenotype conductances from
// ttp06_phenotype_constants.py:54-61.
//
// The kinetics are written once over a number type T: F1 (one cell) or F2
// (two cells packed in a 64-bit register pair, advanced by the sm_100
// packed-FP32 instructions add/sub/mul/fma.rn.ftz.f32x2, which issue once
// for both cells).  Every arithmetic operation is an explicit instruction
// with the same rounding in both types (no compiler contraction or
// reassociation), so a cell gives bit-identical results whichever type, and
// whichever kernel, advances it.  Special functions run per lane.
//
// Differences from the reference are arithmetic only:
//   * FP32 instead of FP64;
//   * constant divisors are folded into multipliers, and exponentials that
//     the reference evaluates twice are shared (exp((V+30)/10) in tau_f and
//     tau_f2; exp((gamma-1) V F/RT) = exp(gamma V F/RT) exp(-V F/RT));
//   * quotients are merged so that each rate needs at most one reciprocal:
//     a product or sum of logistic terms is written over a common
//     denominator, the Rush-Larsen factor exp(-dt/tau) is formed from dt/tau
//     directly where 1/tau is a sum of rates (h, j) or a product of logistic
//     denominators (m, Xr1, Xr2), log(a/b) is log(a) - log(b) with the
//     constant's logarithm folded, and buffer factors 1/(1 + B K/(c+K)^2)
//     are (c+K)^2 / ((c+K)^2 + B K);
//   * exp2V - 1 in I_CaL is evaluated as expm1 (the Taylor series near 0,
//     expm1_t), which is the same quantity with less cancellation near
//     V = 15 mV (the reference's FP64 has the digits to spare; FP32 does
//     not), and exp2V as that plus one;
//   * the special-function unit (SFU) and the FMA pipe share the
//     exponentials: those of the Rush-Larsen factors (unbounded arguments)
//     and of the K1 current (arguments through E_K) use the SFU's base-2
//     exponential; those whose argument is linear or quadratic in V, which
//     the step keeps in [-150, 80] mV so that the argument stays within
//     +-100 in base 2, use exp_fma: 2^x = 2^n 2^f with n = rint(x), f in
//     [-1/2, 1/2], 2^f by a degree-5 polynomial fitted to the relative
//     error on Chebyshev nodes (max relative error 2.1e-7 in FP32, the
//     order of the SFU's approximate exponential), 2^n added to the
//     exponent field.  Reciprocals, logarithms and the square root use the
//     SFU's approximate forms (the same as fast-math division).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace hp {

// state variable order (gpu_ttp06.py:172-176)
enum StateVar : int {
  S_KI = 0, S_NAI, S_CAI, S_XR1, S_XR2, S_XS, S_M, S_H, S_J, S_D, S_F, S_F2,
  S_FCASS, S_S, S_R, S_CASR, S_RPRIME, S_CASS, N_STATE
};

struct CellParams {
  float g_Ks;
  float g_to;
  float g_Kr;
  int endo_s;  // 1 = endo/M-cell s-gate, 0 = epi s-gate
};

// All 18 state variables of one cell, in registers.
struct CellState {
  float v[N_STATE];
};

// ---------------------------------------------------------------------------
// Number types.  F1: one cell.  F2: two cells, lane 0 in the low word.
struct F1 {
  float x;
};
struct F2 {
  unsigned long long x;
};

__device__ __forceinline__ F2 pack2(float a, float b) {
  F2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r.x) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ float lane(F1 v, int) { return v.x; }
__device__ __forceinline__ float lane(F2 v, int l) {
  float a, b;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v.x));
  return l ? b : a;
}
__device__ __forceinline__ void set_lane(F1& v, int, float a) { v.x = a; }
__device__ __forceinline__ void set_lane(F2& v, int l, float a) {
  v = l ? pack2(lane(v, 0), a) : pack2(a, lane(v, 1));
}

template <class T> __device__ __forceinline__ T bc(float c);
template <> __device__ __forceinline__ F1 bc<F1>(float c) { return F1{c}; }
template <> __device__ __forceinline__ F2 bc<F2>(float c) { return pack2(c, c); }

template <class T> struct Lanes;
template <> struct Lanes<F1> { static constexpr int n = 1; };
template <> struct Lanes<F2> { static constexpr int n = 2; };

// rounded-to-nearest, flush-to-zero arithmetic, one instruction each
__device__ __forceinline__ F1 operator+(F1 a, F1 b) {
  F1 r;
  asm("add.rn.ftz.f32 %0, %1, %2;" : "=f"(r.x) : "f"(a.x), "f"(b.x));
  return r;
}
__device__ __forceinline__ F1 operator-(F1 a, F1 b) {
  F1 r;
  asm("sub.rn.ftz.f32 %0, %1, %2;" : "=f"(r.x) : "f"(a.x), "f"(b.x));
  return r;
}
__device__ __forceinline__ F1 operator*(F1 a, F1 b) {
  F1 r;
  asm("mul.rn.ftz.f32 %0, %1, %2;" : "=f"(r.x) : "f"(a.x), "f"(b.x));
  return r;
}
__device__ __forceinline__ F1 fma(F1 a, F1 b, F1 c) {
  F1 r;
  asm("fma.rn.ftz.f32 %0, %1, %2, %3;" : "=f"(r.x) : "f"(a.x), "f"(b.x), "f"(c.x));
  return r;
}
__device__ __forceinline__ F2 operator+(F2 a, F2 b) {
  F2 r;
  asm("add.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r.x) : "l"(a.x), "l"(b.x));
  return r;
}
__device__ __forceinline__ F2 operator-(F2 a, F2 b) {
  F2 r;
  asm("sub.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r.x) : "l"(a.x), "l"(b.x));
  return r;
}
__device__ __forceinline__ F2 operator*(F2 a, F2 b) {
  F2 r;
  asm("mul.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r.x) : "l"(a.x), "l"(b.x));
  return r;
}
__device__ __forceinline__ F2 fma(F2 a, F2 b, F2 c) {
  F2 r;
  asm("fma.rn.ftz.f32x2 %0, %1, %2, %3;" : "=l"(r.x) : "l"(a.x), "l"(b.x), "l"(c.x));
  return r;
}
// mixed with float constants (broadcast to every lane); F1 and F2 only
template <class T> struct IsNum {};
template <> struct IsNum<F1> { using type = F1; };
template <> struct IsNum<F2> { using type = F2; };
template <class T> __device__ __forceinline__ typename IsNum<T>::type operator+(T a, float b) {
  return a + bc<T>(b);
}
template <class T> __device__ __forceinline__ typename IsNum<T>::type operator+(float a, T b) {
  return bc<T>(a) + b;
}
template <class T> __device__ __forceinline__ typename IsNum<T>::type operator-(T a, float b) {
  return a - bc<T>(b);
}
template <class T> __device__ __forceinline__ typename IsNum<T>::type operator-(float a, T b) {
  return bc<T>(a) - b;
}
template <class T> __device__ __forceinline__ typename IsNum<T>::type operator*(T a, float b) {
  return a * bc<T>(b);
}
template <class T> __device__ __forceinline__ typename IsNum<T>::type operator*(float a, T b) {
  return bc<T>(a) * b;
}
template <class T> __device__ __forceinline__ typename IsNum<T>::type operator-(T a) {
  return bc<T>(0.0f) - a;
}

// per-lane functions
template <class T, class Fn>
__device__ __forceinline__ T map1(T a, Fn fn) {
  T r;
#pragma unroll
  for (int l = 0; l < Lanes<T>::n; ++l) set_lane(r, l, fn(lane(a, l)));
  return r;
}
template <class T, class Fn>
__device__ __forceinline__ T map2(T a, T b, Fn fn) {
  T r;
#pragma unroll
  for (int l = 0; l < Lanes<T>::n; ++l) set_lane(r, l, fn(lane(a, l), lane(b, l)));
  return r;
}
__device__ __forceinline__ float sfu_ex2(float x) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float sfu_lg2(float x) {
  float r;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float sfu_rcp(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float sfu_rsqrt(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

constexpr float LOG2E_F = 1.4426950408889634f;
constexpr float LN2_F = 0.6931471805599453f;

template <class T> __device__ __forceinline__ T rcp(T a) { return map1(a, sfu_rcp); }
template <class T> __device__ __forceinline__ T rsqrt(T a) { return map1(a, sfu_rsqrt); }
template <class T> __device__ __forceinline__ T vmin(T a, float c) {
  return map1(a, [c](float x) { return fminf(x, c); });
}
template <class T> __device__ __forceinline__ T vmax(T a, float c) {
  return map1(a, [c](float x) { return fmaxf(x, c); });
}
// a / b with the SFU reciprocal
template <class T> __device__ __forceinline__ T div(T a, T b) { return a * rcp(b); }
template <class T> __device__ __forceinline__ T div(float a, T b) { return a * rcp(b); }

// exp on the SFU (base-2 exponential of x log2 e)
template <class T> __device__ __forceinline__ T exp_sfu(T x) {
  return map1(x * LOG2E_F, sfu_ex2);
}
// natural logarithm on the SFU
template <class T> __device__ __forceinline__ T log_sfu(T x) {
  return map1(x, sfu_lg2) * LN2_F;
}

// exp on the FMA pipe, for |x log2 e| <= 126: 2^y = 2^n 2^f, n = rint(y)
// by the 1.5 * 2^23 shift, f = y - n exact, 2^f by a degree-5 polynomial
// (coefficients fitted to the relative error of 2^f on [-1/2, 1/2]); 2^n is
// added to the exponent field of the polynomial's value.
__device__ __forceinline__ float exp2_scale(float p, float t) {
  return __uint_as_float(__float_as_uint(p) + (__float_as_uint(t) << 23));
}
#ifndef HP_EXP_FMA
#define HP_EXP_FMA 1
#endif
template <class T> __device__ __forceinline__ T exp_fma(T x) {
#if !HP_EXP_FMA
  return exp_sfu(x);
#endif
  constexpr float SHIFT = 12582912.0f;  // 1.5 * 2^23
  const T y = x * LOG2E_F;
  const T t = y + SHIFT;
  const T f = y - (t - SHIFT);
  T p = fma(f, bc<T>(1.3276466634124517e-3f), bc<T>(9.675540961325169e-3f));
  p = fma(p, f, bc<T>(5.550713464617729e-2f));
  p = fma(p, f, bc<T>(2.4022120237350464e-1f));
  p = fma(p, f, bc<T>(6.931469440460205e-1f));
  p = fma(p, f, bc<T>(1.0000001192092896f));
  return map2(p, t, exp2_scale);
}

// exp(x) - 1 without cancellation near 0: the Taylor series to x^8 for
// |x| <= 1/2 (truncation below 1.1e-8 relative), exp(x) - 1 beyond (the
// difference then loses at most a factor 2.6 of relative accuracy).
template <class T> __device__ __forceinline__ T expm1_t(T x) {
  T q = fma(x, bc<T>(1.0f / 40320.0f), bc<T>(1.0f / 5040.0f));
  q = fma(q, x, bc<T>(1.0f / 720.0f));
  q = fma(q, x, bc<T>(1.0f / 120.0f));
  q = fma(q, x, bc<T>(1.0f / 24.0f));
  q = fma(q, x, bc<T>(1.0f / 6.0f));
  q = fma(q, x, bc<T>(0.5f));
  const T small = fma(q * x, x, x);
  const T big = exp_fma(x) - 1.0f;
  T r;
#pragma unroll
  for (int l = 0; l < Lanes<T>::n; ++l)
    set_lane(r, l, fabsf(lane(x, l)) <= 0.5f ? lane(small, l) : lane(big, l));
  return r;
}

// Rush-Larsen update with the exponent given as dt/tau.
template <class T> __device__ __forceinline__ T rl_gate(T x, T xinf, T dt_over_tau) {
  return xinf - (xinf - x) * exp_sfu(-dt_over_tau);
}
// 1 / (1 + exp(x)), the exponential on the FMA pipe
template <class T> __device__ __forceinline__ T sig(T x) { return rcp(1.0f + exp_fma(x)); }

// lane masks
template <class T> struct Mask;
template <> struct Mask<F1> { bool m; };
template <> struct Mask<F2> { bool m0, m1; };
__device__ __forceinline__ Mask<F1> lt(F1 a, float c) { return {a.x < c}; }
__device__ __forceinline__ Mask<F2> lt(F2 a, float c) { return {lane(a, 0) < c, lane(a, 1) < c}; }
__device__ __forceinline__ bool any(Mask<F1> m) { return m.m; }
__device__ __forceinline__ bool all(Mask<F1> m) { return m.m; }
__device__ __forceinline__ bool any(Mask<F2> m) { return m.m0 || m.m1; }
__device__ __forceinline__ bool all(Mask<F2> m) { return m.m0 && m.m1; }
__device__ __forceinline__ F1 sel(Mask<F1> m, F1 a, F1 b) { return m.m ? a : b; }
__device__ __forceinline__ F2 sel(Mask<F2> m, F2 a, F2 b) {
  return pack2(m.m0 ? lane(a, 0) : lane(b, 0), m.m1 ? lane(a, 1) : lane(b, 1));
}

template <class T>
struct CellParamsT {
  T g_Ks, g_to, g_Kr;
  Mask<T> endo_s;  // endo/M-cell s-gate per lane
};
template <class T>
struct CellStateT {
  T v[N_STATE];
};

// Advances `c` by dt at membrane voltage V (one value per lane); returns
// I_ion [mV/ms] per lane.
template <class T>
__device__ __forceinline__ T ttp06_step_t(T V, CellStateT<T>& c, float dt,
                                          const CellParamsT<T>& p) {
  // physical constants (gpu_ttp06.py:95-147)
  constexpr double Rg = 8314.472, Tk = 310.0, Fc = 96485.3415;
  constexpr float RTF = (float)(Rg * Tk / Fc);
  constexpr float FRT = (float)(Fc / (Rg * Tk));
  constexpr float Cao = 2.0f;
  constexpr float g_Na = 14.838f, g_K1 = 5.405f, g_bna = 0.00029f, g_bca = 0.000592f;
  constexpr float g_pCa = 0.1238f, g_pK = 0.0146f, P_NaK = 2.724f, K_mk = 1.0f, Ko = 5.4f;
  constexpr float K_mNa = 40.0f, K_NaCa = 1000.0f, K_sat = 0.1f, alpha_ = 2.5f;
  constexpr float gamma_ = 0.35f, P_kna = 0.03f;
  constexpr float K_pCa = 0.0005f;
  constexpr float k1p = 0.15f, k2p = 0.045f, k3 = 0.06f, k4 = 0.005f, EC = 1.5f;
  constexpr float max_sr = 2.5f, min_sr = 1.0f, V_rel = 0.102f, V_xfer = 0.0038f;
  constexpr float K_up = 0.00025f, V_leak = 0.00036f, Vmax_up = 0.006375f;
  constexpr float Buf_c = 0.2f, K_buf_c = 0.001f, Buf_sr = 10.0f, K_buf_sr = 0.3f;
  constexpr float Buf_ss = 0.4f, K_buf_ss = 0.00025f;
  constexpr double V_c = 0.016404, V_sr = 0.001094, V_ss = 0.00005468;
  constexpr float g_CaL = 3.98e-5f;
  // derived constants
  constexpr float inv_VcF = (float)(1.0 / (V_c * Fc));
  constexpr float inv_2VcF = (float)(1.0 / (2.0 * V_c * Fc));
  constexpr float inv_2VssF = (float)(1.0 / (2.0 * V_ss * Fc));
  constexpr float Vsr_Vc = (float)(V_sr / V_c);
  constexpr float Vsr_Vss = (float)(V_sr / V_ss);
  constexpr float Vc_Vss = (float)(V_c / V_ss);
  constexpr float CaL_k = (float)(4.0 * Fc * Fc / (Rg * Tk));
  constexpr float NaCa_den =
      (float)((87.5 * 87.5 * 87.5 + 140.0 * 140.0 * 140.0) * (1.38 + 2.0));
  constexpr float Nao3 = 140.0f * 140.0f * 140.0f;
  constexpr float NaK_k = P_NaK * Ko / (Ko + K_mk);
  // logarithms of Nao = 140, Ko = 5.4, Ko + P_kna Nao = 9.6 and Cao = 2 (mM)
  constexpr float LN_NAO = 4.941642422609304f, LN_KO = 1.6863989535702288f;
  constexpr float LN_KS = 2.2617630984737906f, LN_CAO = 0.6931471805599453f;
  // sqrt(Ko / 5.4) == 1 for Ko = 5.4

  const T Ki = c.v[S_KI], Nai = c.v[S_NAI], Cai = c.v[S_CAI], Cass = c.v[S_CASS];
  const T CaSR = c.v[S_CASR], Xr1 = c.v[S_XR1], Xr2 = c.v[S_XR2], Xs = c.v[S_XS];
  const T m = c.v[S_M], h = c.v[S_H], j = c.v[S_J], d = c.v[S_D], f = c.v[S_F];
  const T f2 = c.v[S_F2], fCass = c.v[S_FCASS], s = c.v[S_S], r = c.v[S_R];
  const T Rp = c.v[S_RPRIME];

  // reversal potentials
  const T E_Na = RTF * (LN_NAO - log_sfu(Nai));
  const T E_K = RTF * (LN_KO - log_sfu(Ki));
  const T E_Ks = RTF * (LN_KS - log_sfu(fma(bc<T>(P_kna), Nai, Ki)));
  const T E_Ca = (0.5f * RTF) * (LN_CAO - log_sfu(Cai));

  // INa.  tau_m = alpha_m beta_m with alpha_m = 1/(1+e_am) and
  // beta_m = 0.1/(1+e_b1) + 0.1/(1+e_b2) = 0.1 (2+e_b1+e_b2) / ((1+e_b1)(1+e_b2))
  T t1 = sig((-56.86f - V) * (1.0f / 9.03f));
  const T m_inf = t1 * t1;
  const T e_am = exp_fma((-60.0f - V) * 0.2f);
  const T e_b1 = exp_fma((V + 35.0f) * 0.2f);
  const T e_b2 = exp_fma((V - 50.0f) * 0.005f);
  const T dtr_m = div(dt * (1.0f + e_am) * (1.0f + e_b1) * (1.0f + e_b2),
                      0.1f * (2.0f + e_b1 + e_b2));
  t1 = sig((V + 71.55f) * (1.0f / 7.43f));
  const T h_inf = t1 * t1;
  // 1/tau_h = alpha_h + beta_h, 1/tau_j = alpha_j + beta_j (+1e-30)
  T rate_h = bc<T>(0.0f), rate_j = bc<T>(0.0f);
  const Mask<T> low = lt(V, -40.0f);
  if (any(low)) {
    const T rh = 0.057f * exp_fma(-(V + 80.0f) * (1.0f / 6.8f)) + 2.7f * exp_fma(0.079f * V) +
                 3.1e5f * exp_fma(0.3485f * V);
    const T ea = exp_fma(0.311f * (V + 79.23f));    // alpha_j = Aj / (1 + ea)
    const T eb = exp_fma(-0.1378f * (V + 40.14f));  // beta_j = Bj / (1 + eb)
    const T Aj = (-25428.0f * exp_fma(0.2444f * V) - 6.948e-6f * exp_fma(-0.04391f * V)) *
                 (V + 37.78f);
    const T Bj = 0.02424f * exp_fma(-0.01052f * V);
    const T rj = div(Aj * (1.0f + eb) + Bj * (1.0f + ea), (1.0f + ea) * (1.0f + eb));
    rate_h = rh;
    rate_j = rj;
  }
  if (!all(low)) {
    const T rh = div(0.77f / 0.13f, 1.0f + exp_fma((V + 10.66f) * (-1.0f / 11.1f)));
    const T rj = div(0.6f * exp_fma(0.057f * V), 1.0f + exp_fma(-0.1f * (V + 32.0f)));
    rate_h = sel(low, rate_h, rh);
    rate_j = sel(low, rate_j, rj);
  }
  const T dtr_h = dt * (rate_h + 1e-30f);
  const T dtr_j = dt * (rate_j + 1e-30f);
  const T i_Na = g_Na * m * m * m * h * j * (V - E_Na);

  // IKr.  tau_xr1 = 2700 / ((1+e_m45)(1+e_x1)), tau_xr2 = 3.36 / ((1+e_x2)(1+e_x3))
  const T xr1_inf = sig((-26.0f - V) * (1.0f / 7.0f));
  const T e_m45 = exp_fma((-45.0f - V) * 0.1f);
  const T e_p30 = exp_fma((V + 30.0f) * 0.1f);  // shared by tau_f, tau_f2
  const T dtr_xr1 = dt * (1.0f + e_m45) * (1.0f + exp_fma((V + 30.0f) * (1.0f / 11.5f))) *
                    (1.0f / 2700.0f);
  const T xr2_inf = sig((V + 88.0f) * (1.0f / 24.0f));
  const T dtr_xr2 = dt * (1.0f + exp_fma((-60.0f - V) * 0.05f)) *
                    (1.0f + exp_fma((V - 60.0f) * 0.05f)) * (1.0f / 3.36f);
  const T i_Kr = p.g_Kr * Xr1 * Xr2 * (V - E_K);

  // IKs.  tau_xs = 1400 q / (1+e) + 80 = (1400 q + 80 (1+e)) / (1+e)
  const T xs_inf = sig((-5.0f - V) * (1.0f / 14.0f));
  const T q_xs = rsqrt(1.0f + exp_fma((5.0f - V) * (1.0f / 6.0f)));
  const T e_xs = exp_fma((V - 35.0f) * (1.0f / 15.0f));
  const T dtr_xs = div(dt * (1.0f + e_xs), 1400.0f * q_xs + 80.0f * (1.0f + e_xs));
  const T i_Ks = p.g_Ks * Xs * Xs * (V - E_Ks);

  // IK1.  xk1 = ak1 / (ak1 + bk1) with ak1 = 0.1/(1+e1), bk1 = nb/(1+e4)
  // = 0.1 (1+e4) / (0.1 (1+e4) + nb (1+e1)); exponents bounded so that the
  // merged form stays finite for any state
  const T VmEK = V - E_K;
  const T e1 = exp_sfu(vmin(0.06f * (VmEK - 200.0f), 80.0f));
  const T nb = 3.0f * exp_sfu(vmin(2e-4f * (VmEK + 100.0f), 80.0f)) +
               exp_sfu(vmin(0.1f * (VmEK - 10.0f), 80.0f));
  const T a4 = 0.1f * (1.0f + exp_sfu(vmin(-0.5f * VmEK, 80.0f)));
  const T xk1_inf = div(a4, a4 + nb * (1.0f + e1));
  const T i_K1 = g_K1 * xk1_inf * VmEK;

  // Ito
  T s_inf = bc<T>(0.0f), dtr_s = bc<T>(0.0f);
  if (any(p.endo_s)) {
    s_inf = sig((V + 28.0f) * 0.2f);
    const T a = V + 67.0f;
    dtr_s = div(bc<T>(dt), 1000.0f * exp_fma(-a * a * 0.001f) + 8.0f);
  }
  if (!all(p.endo_s)) {
    // tau_s = g + 5/(1+e) + 3 = ((g+3)(1+e) + 5) / (1+e)
    const T si = sig((V + 20.0f) * 0.2f);
    const T a = V + 45.0f;
    const T g = 85.0f * exp_fma(-a * a * (1.0f / 320.0f));
    const T e = exp_fma((V - 20.0f) * 0.2f);
    const T ds = div(dt * (1.0f + e), (g + 3.0f) * (1.0f + e) + 5.0f);
    s_inf = sel(p.endo_s, s_inf, si);
    dtr_s = sel(p.endo_s, dtr_s, ds);
  }
  const T r_inf = sig((20.0f - V) * (1.0f / 6.0f));
  const T a40 = V + 40.0f;
  const T dtr_r = div(bc<T>(dt), 9.5f * exp_fma(-a40 * a40 * (1.0f / 1800.0f)) + 0.8f);
  const T i_to = p.g_to * r * s * VmEK;

  // ICaL.  tau_d = (1.4/(1+ea) + 0.25) 1.4/(1+eb) + 1/(1+ec)
  //        = (1.4 (1.4 + 0.25 (1+ea)) (1+ec) + (1+ea)(1+eb)) / ((1+ea)(1+eb)(1+ec))
  const T d_inf = sig((-8.0f - V) * (1.0f / 7.5f));
  const T ea_d = 1.0f + exp_fma((-35.0f - V) * (1.0f / 13.0f));
  const T eb_d = 1.0f + exp_fma((V + 5.0f) * 0.2f);
  const T ec_d = 1.0f + exp_fma((50.0f - V) * 0.05f);
  const T P_d = ea_d * eb_d;
  const T dtr_d = div(dt * P_d * ec_d, 1.4f * (1.4f + 0.25f * ea_d) * ec_d + P_d);
  // tau_f = G + 200/(1+eA) + 180/(1+eB) + 20, over the denominator (1+eA)(1+eB)
  const T f_inf = sig((V + 20.0f) * (1.0f / 7.0f));
  const T a27 = V + 27.0f;
  const T eB = 1.0f + e_p30;
  const T eA = 1.0f + exp_fma((13.0f - V) * 0.1f);
  const T D_f = eA * eB;
  const T dtr_f = div(dt * D_f, (1102.5f * exp_fma(-a27 * a27 * (1.0f / 225.0f)) + 20.0f) * D_f +
                                    200.0f * eB + 180.0f * eA);
  // tau_f2 = G2 + 31/(1+eC) + 80/(1+eB)
  const T f2_inf = 0.67f * sig((V + 35.0f) * (1.0f / 7.0f)) + 0.33f;
  const T eC = 1.0f + exp_fma((25.0f - V) * 0.1f);
  const T D_f2 = eC * eB;
  const T dtr_f2 = div(dt * D_f2, 562.0f * exp_fma(-a27 * a27 * (1.0f / 240.0f)) * D_f2 +
                                      31.0f * eB + 80.0f * eC);
  // fCass: inf = 0.6/(1+cq) + 0.4, tau = 80/(1+cq) + 2 = (82 + 2 cq)/(1+cq)
  const T c20 = Cass * 20.0f;
  const T cq = c20 * c20;
  const T fCass_inf = div(0.6f, 1.0f + cq) + 0.4f;
  const T dtr_fCass = div(dt * (1.0f + cq), 82.0f + 2.0f * cq);

  const T x2v = 2.0f * (V - 15.0f) * FRT;
  T denom = expm1_t(x2v);
  const T exp2V = denom + 1.0f;
  denom = map1(denom, [](float x) { return fabsf(x) < 1e-10f ? 1e-10f : x; });
  const T i_CaL = div(g_CaL * d * f * f2 * fCass * CaL_k * (V - 15.0f) *
                          (0.25f * Cass * exp2V - Cao),
                      denom);

  // background, pump, exchanger
  const T i_bNa = g_bna * (V - E_Na);
  const T i_bCa = g_bca * (V - E_Ca);
  const T i_pCa = div(g_pCa * Cai, Cai + K_pCa);
  const T i_pK = g_pK * VmEK * sig((25.0f - V) * (1.0f / 5.98f));
  const T VF = V * FRT;
  const T e_mVF = exp_fma(-VF);
  const T i_NaK = div(NaK_k * Nai, (Nai + K_mNa) * (1.0f + 0.1245f * exp_fma(-0.1f * VF) +
                                                    0.0353f * e_mVF));
  const T eVg = exp_fma(gamma_ * VF);
  const T eVgm1 = eVg * e_mVF;  // exp((gamma - 1) V F / RT)
  const T i_NaCa = div(K_NaCa * (eVg * Nai * Nai * Nai * Cao - eVgm1 * Nao3 * Cai * alpha_),
                       NaCa_den * (1.0f + K_sat * eVgm1));

  const T I_ion = i_K1 + i_to + i_Kr + i_Ks + i_CaL + i_NaK + i_Na + i_bNa + i_NaCa +
                  i_bCa + i_pCa + i_pK;

  // SR calcium.  kcasr = max - (max-min) CaSR^2 / (CaSR^2 + EC^2);
  // O = k1 Cass^2 R' / (k3 + k1 Cass^2) with k1 = k1p / kcasr
  const T CaSR2 = CaSR * CaSR;
  const T kcasr = max_sr - div((max_sr - min_sr) * CaSR2, CaSR2 + EC * EC);
  const T k2 = k2p * kcasr;
  const T Cass2 = Cass * Cass;
  const T O = div(k1p * Cass2 * Rp, k3 * kcasr + k1p * Cass2);
  const T i_rel = V_rel * O * (CaSR - Cass);
  const T c2 = Cai * Cai + 1e-30f;
  const T i_up = div(Vmax_up * c2, c2 + K_up * K_up);
  const T i_leak = V_leak * (CaSR - Cai);
  const T i_xfer = V_xfer * (Cass - Cai);
  const T bcc = Cai + K_buf_c, bsr = CaSR + K_buf_sr, bss = Cass + K_buf_ss;
  const T bufc = div(bcc * bcc, bcc * bcc + Buf_c * K_buf_c);
  const T bufsr = div(bsr * bsr, bsr * bsr + Buf_sr * K_buf_sr);
  const T bufss = div(bss * bss, bss * bss + Buf_ss * K_buf_ss);

  const T dNai = -(i_Na + i_bNa + 3.0f * i_NaK + 3.0f * i_NaCa) * inv_VcF;
  const T dKi = -(i_K1 + i_to + i_Kr + i_Ks + i_pK - 2.0f * i_NaK) * inv_VcF;
  const T dCai = bufc * ((i_leak - i_up) * Vsr_Vc + i_xfer -
                         (i_bCa + i_pCa - 2.0f * i_NaCa) * inv_2VcF);
  const T dCaSR = bufsr * (i_up - i_rel - i_leak);
  const T dCass = bufss * (-i_CaL * inv_2VssF + i_rel * Vsr_Vss - i_xfer * Vc_Vss);

  c.v[S_M] = rl_gate(m, m_inf, dtr_m);
  c.v[S_H] = rl_gate(h, h_inf, dtr_h);
  c.v[S_J] = rl_gate(j, h_inf, dtr_j);
  c.v[S_XR1] = rl_gate(Xr1, xr1_inf, dtr_xr1);
  c.v[S_XR2] = rl_gate(Xr2, xr2_inf, dtr_xr2);
  c.v[S_XS] = rl_gate(Xs, xs_inf, dtr_xs);
  c.v[S_D] = rl_gate(d, d_inf, dtr_d);
  c.v[S_F] = rl_gate(f, f_inf, dtr_f);
  c.v[S_F2] = rl_gate(f2, f2_inf, dtr_f2);
  c.v[S_FCASS] = rl_gate(fCass, fCass_inf, dtr_fCass);
  c.v[S_S] = rl_gate(s, s_inf, dtr_s);
  c.v[S_R] = rl_gate(r, r_inf, dtr_r);
  c.v[S_RPRIME] = Rp + dt * (-k2 * Cass * Rp + k4 * (1.0f - Rp));
  c.v[S_NAI] = vmax(fma(bc<T>(dt), dNai, Nai), 1e-3f);
  c.v[S_KI] = vmax(fma(bc<T>(dt), dKi, Ki), 1e-3f);
  c.v[S_CAI] = vmax(fma(bc<T>(dt), dCai, Cai), 1e-7f);
  c.v[S_CASR] = vmax(fma(bc<T>(dt), dCaSR, CaSR), 1e-7f);
  c.v[S_CASS] = vmax(fma(bc<T>(dt), dCass, Cass), 1e-7f);
  return I_ion;
}

// W = V + dt/Cm (-I_ion Cm + I_stim), two explicit FMAs (every kernel forms
// the ionic half's output with this one expression).
__device__ __forceinline__ float w_update(float V, float Iion, float Istim, float dt_over_Cm,
                                          float Cm) {
  const F1 t = fma(F1{-Iion}, F1{Cm}, F1{Istim});
  return fma(F1{dt_over_Cm}, t, F1{V}).x;
}

// One cell (the fused kernels, Purkinje nodes).
__device__ __forceinline__ float ttp06_step(float V, CellState& c, float dt, const CellParams p) {
  CellStateT<F1> s;
#pragma unroll
  for (int v = 0; v < N_STATE; ++v) s.v[v] = F1{c.v[v]};
  CellParamsT<F1> q{F1{p.g_Ks}, F1{p.g_to}, F1{p.g_Kr}, Mask<F1>{p.endo_s != 0}};
  const F1 I = ttp06_step_t<F1>(F1{V}, s, dt, q);
#pragma unroll
  for (int v = 0; v < N_STATE; ++v) c.v[v] = s.v[v].x;
  return I.x;
}

// Two cells at once (lanes 0 and 1), with their own phenotype parameters.
__device__ __forceinline__ F2 ttp06_step2(F2 V, CellStateT<F2>& c, float dt, const CellParams p0,
                                          const CellParams p1) {
  CellParamsT<F2> q{pack2(p0.g_Ks, p1.g_Ks), pack2(p0.g_to, p1.g_to), pack2(p0.g_Kr, p1.g_Kr),
                    Mask<F2>{p0.endo_s != 0, p1.endo_s != 0}};
  return ttp06_step_t<F2>(V, c, dt, q);
}

}  // namespace hp
