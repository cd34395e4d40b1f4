// TTP06 (ten Tusscher & Panfilov 2006) single-cell update in FP32, one
// thread per cell.  Same kinetics as HrdayaPy's
// simulation/functions/ionic_models/gpu_ttp06.py:198-412 (_currents_and_gates):
// Rush-Larsen for the 12 gates, forward Euler for Rprime and the five
// concentrations with the reference's clamps, phenotype conductances from
// ttp06_phenotype_constants.py:54-61.
//
// Differences from the reference are arithmetic only:
//   * FP32 instead of FP64;
//   * constant divisors are folded into multipliers, and exponentials that
//     the reference evaluates twice are shared (exp((V+30)/10) in tau_f and
//     tau_f2; exp((gamma-1) V F/RT) = exp(gamma V F/RT) exp(-V F/RT));
//   * quotients are merged so that each rate needs at most one reciprocal
//     (the special-function unit is the scarce pipe of this kernel): a
//     product or sum of logistic terms is written over a common denominator,
//     the Rush-Larsen factor exp(-dt/tau) is formed from dt/tau directly
//     where 1/tau is a sum of rates (h, j) or a product of logistic
//     denominators (m, Xr1, Xr2), log(a/b) is log(a) - log(b) with the
//     constant's logarithm folded, and buffer factors 1/(1 + B K/(c+K)^2)
//     are (c+K)^2 / ((c+K)^2 + B K);
//   * exponentials of V with a common slope a share one exp(a V):
//     exp(a (V + c)) = exp(a c) exp(a V) for the slopes 1/5, +-1/10,
//     +-1/20, 1/7 and -1/6 (seven exponentials instead of eighteen), and a
//     logistic 1 / (1 + exp(a c) / E) is E / (E + exp(a c));
//   * exp2V - 1 in I_CaL is evaluated with expm1f, which is the same
//     quantity with less cancellation near V = 15 mV (the reference's FP64
//     has the digits to spare; FP32 does not), and exp2V as that plus one.
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

// Exponential / logarithm used by the kinetics.  HP_FAST_EXP selects the
// SFU intrinsics (__expf/__logf); otherwise the accurate libdevice versions.
#ifdef HP_FAST_EXP
__device__ __forceinline__ float hexp(float x) { return __expf(x); }
__device__ __forceinline__ float hlog(float x) { return __logf(x); }
#else
__device__ __forceinline__ float hexp(float x) { return expf(x); }
__device__ __forceinline__ float hlog(float x) { return logf(x); }
#endif

// Rush-Larsen update with the exponent given as dt/tau.
__device__ __forceinline__ float rl_gate(float x, float xinf, float dt_over_tau) {
  return xinf - (xinf - x) * hexp(-dt_over_tau);
}

__device__ __forceinline__ float sig(float x) {  // 1 / (1 + exp(x))
  return 1.0f / (1.0f + hexp(x));
}

// Advances `c` by dt at membrane voltage V; returns I_ion [mV/ms].
__device__ __forceinline__ float ttp06_step(float V, CellState& c, float dt,
                                            const CellParams p) {
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
  constexpr float sqko = 1.0f;
  // exp(c) for the offsets of the exponentials that share a slope (below)
  constexpr float X_M12 = (float)6.14421235332821e-06, X_7 = (float)1096.6331584284585;
  constexpr float X_1 = (float)2.718281828459045, X_56 = (float)270.42640742615254;
  constexpr float X_4 = (float)54.598150033144236, X_M4 = (float)0.01831563888873418;
  constexpr float X_M45 = (float)0.011108996538242306, X_3 = (float)20.085536923187668;
  constexpr float X_13 = (float)3.6692966676192444, X_25 = (float)12.182493960703473;
  constexpr float X_M32 = (float)0.04076220397836621, X_M3 = (float)0.049787068367863944;
  constexpr float X_M26_7 = (float)0.0243728440732796, X_20_7 = (float)17.41170806332765;
  constexpr float X_5 = (float)148.4131591025766, X_5_6 = (float)2.300975890892825;
  constexpr float X_10_3 = (float)28.03162489452614;

  const float Ki = c.v[S_KI], Nai = c.v[S_NAI], Cai = c.v[S_CAI], Cass = c.v[S_CASS];
  const float CaSR = c.v[S_CASR], Xr1 = c.v[S_XR1], Xr2 = c.v[S_XR2], Xs = c.v[S_XS];
  const float m = c.v[S_M], h = c.v[S_H], j = c.v[S_J], d = c.v[S_D], f = c.v[S_F];
  const float f2 = c.v[S_F2], fCass = c.v[S_FCASS], s = c.v[S_S], r = c.v[S_R];
  const float Rp = c.v[S_RPRIME];

  // reversal potentials
  const float E_Na = RTF * (LN_NAO - hlog(Nai));
  const float E_K = RTF * (LN_KO - hlog(Ki));
  const float E_Ks = RTF * (LN_KS - hlog(Ki + P_kna * Nai));
  const float E_Ca = (0.5f * RTF) * (LN_CAO - hlog(Cai));

  // Exponentials of V that share a slope a are formed once:
  // exp(a (V + c)) = exp(a c) exp(a V), with exp(a c) a constant.  A logistic
  // 1 / (1 + K / E) is written E / (E + K), inside its one reciprocal.
  const float P2 = hexp(0.2f * V);              // exp(V / 5)
  const float Em1 = hexp(-0.1f * V);            // exp(-V / 10)
  const float Ep1 = hexp(0.1f * V);             // exp(V / 10)
  const float P05 = hexp(0.05f * V);            // exp(V / 20)
  const float M05 = hexp(-0.05f * V);           // exp(-V / 20)
  const float P7 = hexp(V * (1.0f / 7.0f));     // exp(V / 7)
  const float M6 = hexp(V * (-1.0f / 6.0f));    // exp(-V / 6)

  // INa.  tau_m = alpha_m beta_m with alpha_m = 1/(1+e_am) and
  // beta_m = 0.1/(1+e_b1) + 0.1/(1+e_b2) = 0.1 (2+e_b1+e_b2) / ((1+e_b1)(1+e_b2));
  // 1 + e_am = 1 + exp(-12) / P2 = (P2 + exp(-12)) / P2
  float t1 = sig((-56.86f - V) * (1.0f / 9.03f));
  const float m_inf = t1 * t1;
  const float e_b1 = X_7 * P2;                  // exp((V + 35) / 5)
  const float e_b2 = hexp((V - 50.0f) * 0.005f);
  const float dtr_m = dt * (P2 + X_M12) * (1.0f + e_b1) * (1.0f + e_b2) /
                      (0.1f * (2.0f + e_b1 + e_b2) * P2);
  t1 = sig((V + 71.55f) * (1.0f / 7.43f));
  const float h_inf = t1 * t1;
  // 1/tau_h = alpha_h + beta_h, 1/tau_j = alpha_j + beta_j (+1e-30)
  float rate_h, rate_j;
  if (V < -40.0f) {
    rate_h = 0.057f * hexp(-(V + 80.0f) * (1.0f / 6.8f)) + 2.7f * hexp(0.079f * V) +
             3.1e5f * hexp(0.3485f * V);
    const float ea = hexp(0.311f * (V + 79.23f));    // alpha_j = Aj / (1 + ea)
    const float eb = hexp(-0.1378f * (V + 40.14f));  // beta_j = Bj / (1 + eb)
    const float Aj = (-25428.0f * hexp(0.2444f * V) - 6.948e-6f * hexp(-0.04391f * V)) *
                     (V + 37.78f);
    const float Bj = 0.02424f * hexp(-0.01052f * V);
    rate_j = (Aj * (1.0f + eb) + Bj * (1.0f + ea)) / ((1.0f + ea) * (1.0f + eb));
  } else {
    rate_h = (0.77f / 0.13f) / (1.0f + hexp((V + 10.66f) * (-1.0f / 11.1f)));
    rate_j = 0.6f * hexp(0.057f * V) / (1.0f + X_M32 * Em1);
  }
  const float dtr_h = dt * (rate_h + 1e-30f);
  const float dtr_j = dt * (rate_j + 1e-30f);
  const float i_Na = g_Na * m * m * m * h * j * (V - E_Na);

  // IKr.  tau_xr1 = 2700 / ((1+e_m45)(1+e_x1)), tau_xr2 = 3.36 / ((1+e_x2)(1+e_x3))
  const float xr1_inf = P7 / (P7 + X_M26_7);    // 1 / (1 + exp((-26 - V) / 7))
  const float e_m45 = X_M45 * Em1;               // exp((-45 - V) / 10)
  const float e_p30 = X_3 * Ep1;                 // exp((V + 30) / 10), shared by tau_f, tau_f2
  const float dtr_xr1 = dt * (1.0f + e_m45) * (1.0f + hexp((V + 30.0f) * (1.0f / 11.5f))) *
                        (1.0f / 2700.0f);
  const float xr2_inf = sig((V + 88.0f) * (1.0f / 24.0f));
  const float dtr_xr2 = dt * (1.0f + X_M3 * M05) * (1.0f + X_M3 * P05) * (1.0f / 3.36f);
  const float i_Kr = p.g_Kr * sqko * Xr1 * Xr2 * (V - E_K);

  // IKs.  tau_xs = 1400 q / (1+e) + 80 = (1400 q + 80 (1+e)) / (1+e)
  const float xs_inf = sig((-5.0f - V) * (1.0f / 14.0f));
  const float q_xs = rsqrtf(1.0f + X_5_6 * M6);  // exp((5 - V) / 6)
  const float e_xs = hexp((V - 35.0f) * (1.0f / 15.0f));
  const float dtr_xs = dt * (1.0f + e_xs) / (1400.0f * q_xs + 80.0f * (1.0f + e_xs));
  const float i_Ks = p.g_Ks * Xs * Xs * (V - E_Ks);

  // IK1.  xk1 = ak1 / (ak1 + bk1) with ak1 = 0.1/(1+e1), bk1 = nb/(1+e4)
  // = 0.1 (1+e4) / (0.1 (1+e4) + nb (1+e1)); exponents bounded so that the
  // merged form stays finite for any state
  const float VmEK = V - E_K;
  const float e1 = hexp(fminf(0.06f * (VmEK - 200.0f), 80.0f));
  const float nb = 3.0f * hexp(fminf(2e-4f * (VmEK + 100.0f), 80.0f)) +
                   hexp(fminf(0.1f * (VmEK - 10.0f), 80.0f));
  const float a4 = 0.1f * (1.0f + hexp(fminf(-0.5f * VmEK, 80.0f)));
  const float xk1_inf = a4 / (a4 + nb * (1.0f + e1));
  const float i_K1 = g_K1 * sqko * xk1_inf * VmEK;

  // Ito
  float s_inf, dtr_s;
  if (p.endo_s) {
    s_inf = 1.0f / (1.0f + X_56 * P2);           // sig((V + 28) / 5)
    const float a = V + 67.0f;
    dtr_s = dt / (1000.0f * hexp(-a * a * 0.001f) + 8.0f);
  } else {
    // tau_s = g + 5/(1+e) + 3 = ((g+3)(1+e) + 5) / (1+e)
    s_inf = 1.0f / (1.0f + X_4 * P2);            // sig((V + 20) / 5)
    const float a = V + 45.0f;
    const float g = 85.0f * hexp(-a * a * (1.0f / 320.0f));
    const float e = X_M4 * P2;                     // exp((V - 20) / 5)
    dtr_s = dt * (1.0f + e) / ((g + 3.0f) * (1.0f + e) + 5.0f);
  }
  const float r_inf = 1.0f / (1.0f + X_10_3 * M6);   // sig((20 - V) / 6)
  const float a40 = V + 40.0f;
  const float dtr_r = dt / (9.5f * hexp(-a40 * a40 * (1.0f / 1800.0f)) + 0.8f);
  const float i_to = p.g_to * r * s * VmEK;

  // ICaL.  tau_d = (1.4/(1+ea) + 0.25) 1.4/(1+eb) + 1/(1+ec)
  //        = (1.4 (1.4 + 0.25 (1+ea)) (1+ec) + (1+ea)(1+eb)) / ((1+ea)(1+eb)(1+ec))
  const float d_inf = sig((-8.0f - V) * (1.0f / 7.5f));
  const float ea_d = 1.0f + hexp((-35.0f - V) * (1.0f / 13.0f));
  const float eb_d = 1.0f + X_1 * P2;            // 1 + exp((V + 5) / 5)
  const float ec_d = 1.0f + X_25 * M05;          // 1 + exp((50 - V) / 20)
  const float P_d = ea_d * eb_d;
  const float dtr_d = dt * P_d * ec_d / (1.4f * (1.4f + 0.25f * ea_d) * ec_d + P_d);
  // tau_f = G + 200/(1+eA) + 180/(1+eB) + 20, over the denominator (1+eA)(1+eB)
  const float f_inf = 1.0f / (1.0f + X_20_7 * P7);  // sig((V + 20) / 7)
  const float a27 = V + 27.0f;
  const float eB = 1.0f + e_p30;
  const float eA = 1.0f + X_13 * Em1;            // 1 + exp((13 - V) / 10)
  const float D_f = eA * eB;
  const float dtr_f = dt * D_f /
                      ((1102.5f * hexp(-a27 * a27 * (1.0f / 225.0f)) + 20.0f) * D_f +
                       200.0f * eB + 180.0f * eA);
  // tau_f2 = G2 + 31/(1+eC) + 80/(1+eB)
  const float f2_inf = 0.67f / (1.0f + X_5 * P7) + 0.33f;   // 0.67 sig((V + 35) / 7) + 0.33
  const float eC = 1.0f + X_25 * Em1;            // 1 + exp((25 - V) / 10)
  const float D_f2 = eC * eB;
  const float dtr_f2 = dt * D_f2 /
                       (562.0f * hexp(-a27 * a27 * (1.0f / 240.0f)) * D_f2 + 31.0f * eB +
                        80.0f * eC);
  // fCass: inf = 0.6/(1+cq) + 0.4, tau = 80/(1+cq) + 2 = (82 + 2 cq)/(1+cq)
  const float cq = (Cass * 20.0f) * (Cass * 20.0f);
  const float fCass_inf = 0.6f / (1.0f + cq) + 0.4f;
  const float dtr_fCass = dt * (1.0f + cq) / (82.0f + 2.0f * cq);

  const float x2v = 2.0f * (V - 15.0f) * FRT;
  float denom = expm1f(x2v);
  const float exp2V = denom + 1.0f;
  if (fabsf(denom) < 1e-10f) denom = 1e-10f;
  const float i_CaL = g_CaL * d * f * f2 * fCass * CaL_k * (V - 15.0f) *
                      (0.25f * Cass * exp2V - Cao) / denom;

  // background, pump, exchanger
  const float i_bNa = g_bna * (V - E_Na);
  const float i_bCa = g_bca * (V - E_Ca);
  const float i_pCa = g_pCa * Cai / (Cai + K_pCa);
  const float i_pK = g_pK * VmEK * sig((25.0f - V) * (1.0f / 5.98f));
  const float VF = V * FRT;
  const float e_mVF = hexp(-VF);
  const float i_NaK = NaK_k * Nai /
                      ((Nai + K_mNa) * (1.0f + 0.1245f * hexp(-0.1f * VF) + 0.0353f * e_mVF));
  const float eVg = hexp(gamma_ * VF);
  const float eVgm1 = eVg * e_mVF;  // exp((gamma - 1) V F / RT)
  const float i_NaCa = K_NaCa * (eVg * Nai * Nai * Nai * Cao - eVgm1 * Nao3 * Cai * alpha_) /
                       (NaCa_den * (1.0f + K_sat * eVgm1));

  const float I_ion = i_K1 + i_to + i_Kr + i_Ks + i_CaL + i_NaK + i_Na + i_bNa + i_NaCa +
                      i_bCa + i_pCa + i_pK;

  // SR calcium.  kcasr = max - (max-min) CaSR^2 / (CaSR^2 + EC^2);
  // O = k1 Cass^2 R' / (k3 + k1 Cass^2) with k1 = k1p / kcasr
  const float CaSR2 = CaSR * CaSR;
  const float kcasr = max_sr - (max_sr - min_sr) * CaSR2 / (CaSR2 + EC * EC);
  const float k2 = k2p * kcasr;
  const float Cass2 = Cass * Cass;
  const float O = k1p * Cass2 * Rp / (k3 * kcasr + k1p * Cass2);
  const float i_rel = V_rel * O * (CaSR - Cass);
  const float c2 = Cai * Cai + 1e-30f;
  const float i_up = Vmax_up * c2 / (c2 + K_up * K_up);
  const float i_leak = V_leak * (CaSR - Cai);
  const float i_xfer = V_xfer * (Cass - Cai);
  const float bc = Cai + K_buf_c, bsr = CaSR + K_buf_sr, bss = Cass + K_buf_ss;
  const float bufc = bc * bc / (bc * bc + Buf_c * K_buf_c);
  const float bufsr = bsr * bsr / (bsr * bsr + Buf_sr * K_buf_sr);
  const float bufss = bss * bss / (bss * bss + Buf_ss * K_buf_ss);

  const float dNai = -(i_Na + i_bNa + 3.0f * i_NaK + 3.0f * i_NaCa) * inv_VcF;
  const float dKi = -(i_K1 + i_to + i_Kr + i_Ks + i_pK - 2.0f * i_NaK) * inv_VcF;
  const float dCai = bufc * ((i_leak - i_up) * Vsr_Vc + i_xfer -
                             (i_bCa + i_pCa - 2.0f * i_NaCa) * inv_2VcF);
  const float dCaSR = bufsr * (i_up - i_rel - i_leak);
  const float dCass = bufss * (-i_CaL * inv_2VssF + i_rel * Vsr_Vss - i_xfer * Vc_Vss);

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
  c.v[S_NAI] = fmaxf(Nai + dt * dNai, 1e-3f);
  c.v[S_KI] = fmaxf(Ki + dt * dKi, 1e-3f);
  c.v[S_CAI] = fmaxf(Cai + dt * dCai, 1e-7f);
  c.v[S_CASR] = fmaxf(CaSR + dt * dCaSR, 1e-7f);
  c.v[S_CASS] = fmaxf(Cass + dt * dCass, 1e-7f);
  return I_ion;
}

}  // namespace hp
