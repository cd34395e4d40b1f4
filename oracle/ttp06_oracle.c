/*
 * ORACLE -- test infrastructure, not product code.
 *
 * FP64 CPU restatement of HrdayaPy's monodomain hot path, used only by the
 * tests, by smoke() as the checker, and as the timed CPU baseline in
 * bench.py.  Nothing in the product (hrdayapy_b200/) links or calls it.
 *
 *   orc_ttp06_cell   one TTP06 (ten Tusscher & Panfilov 2006) update of one
 *                    cell: Rush-Larsen gates, forward-Euler Rprime and
 *                    concentrations with the reference's clamps.  Follows
 *                    hrdayapy/simulation/functions/ionic_models/gpu_ttp06.py
 *                    :198-412 (_currents_and_gates) term by term, with the
 *                    phenotype table of ttp06_phenotype_constants.py:54-61.
 *   orc_mono_run     the Lie-split time loop of run_coupled
 *                    (purkinje_myocardium_pipeline.py:1347-1420) and of the
 *                    anisotropic solver (..._anisotropic_solver.py:1746-1820)
 *                    at theta = 0: ionic step on V^n, V* = V + dt/Cm (-Iion Cm
 *                    + Istim), V^{n+1} = clamp(V* + dt/Cm L V*, -150, 80),
 *                    where L = D^-1 K is the assembled global Laplacian (CSR).
 *                    At theta = 0 the reference's BiCGSTAB on
 *                    A = (Cm/dt) I converges in one iteration to exactly this
 *                    update (pipeline.py:691-754).
 *
 * Build: make -C oracle   (gcc -O2 -pthread, no fast-math: IEEE FP64).
 * Work is split over a pthread team in static node slices; every node's
 * arithmetic is independent of the split, so results do not depend on the
 * thread count.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#include <stdlib.h>
#include <pthread.h>
#include <unistd.h>

/* state column order, gpu_ttp06.py:172-176 */
enum { KI = 0, NAI, CAI, XR1, XR2, XS, M_, H_, J_, D_, F_, F2_, FCASS, S_, R_,
       CASR, RPRIME, CASS, NSTATE };

/* gpu_ttp06.py:95-147 */
static const double Rgas = 8314.472, Tk = 310.0, F_c = 96485.3415;
#define RTF (Rgas * Tk / F_c)
#define FRT (F_c / (Rgas * Tk))
static const double Ko = 5.4, Nao = 140.0, Cao = 2.0;
static const double g_Na = 14.838, g_K1 = 5.405, g_bna = 0.00029, g_bca = 0.000592,
                    g_pCa = 0.1238, g_pK = 0.0146, P_NaK = 2.724, K_mk = 1.0,
                    K_mNa = 40.0, K_NaCa = 1000.0, K_sat = 0.1, alpha_ = 2.5,
                    gamma_ = 0.35, Km_Ca = 1.38, Km_Nai = 87.5, P_kna = 0.03,
                    K_pCa = 0.0005;
static const double k1p = 0.15, k2p = 0.045, k3 = 0.06, k4 = 0.005, EC = 1.5,
                    max_sr = 2.5, min_sr = 1.0, V_rel = 0.102, V_xfer = 0.0038,
                    K_up = 0.00025, V_leak = 0.00036, Vmax_up = 0.006375,
                    Buf_c = 0.2, K_buf_c = 0.001, Buf_sr = 10.0, K_buf_sr = 0.3,
                    Buf_ss = 0.4, K_buf_ss = 0.00025, V_c = 0.016404,
                    V_sr = 0.001094, V_ss = 0.00005468, Cm_model = 1.0;

/* ttp06_phenotype_constants.py:54-61: 0 endo, 1 mid, 2 epi */
static const double PH_GKS[3] = {0.392, 0.098, 0.392};
static const double PH_GTO[3] = {0.073, 0.294, 0.294};
static const int PH_ENDO_S[3] = {1, 1, 0};
static const double G_KR = 0.153, G_CAL = 3.98e-5;

/* gpu_ttp06.py:150-169 */
void orc_ttp06_init(double *st) {
    static const double init[NSTATE] = {138.4, 10.355, 0.00013, 0.00448, 0.476,
        0.0087, 0.00155, 0.7573, 0.7225, 3.164e-5, 0.8009, 0.9778, 0.9953,
        0.3212, 2.235e-8, 3.715, 0.9068, 0.00036};
    memcpy(st, init, sizeof(init));
}

static inline double rl(double x, double xinf, double tau, double dt) {
    return xinf - (xinf - x) * exp(-dt / tau);
}

/* One cell.  st: 18 states (updated in place).  Returns I_ion [mV/ms].
 * gks_s / gkr_s scale the phenotype's g_Ks / g_Kr (1.0 = reference). */
double orc_ttp06_cell(double V, double *st, double dt, int pheno,
                      double gks_s, double gkr_s) {
    const double g_Ks = PH_GKS[pheno] * gks_s, g_to = PH_GTO[pheno];
    const double g_Kr = G_KR * gkr_s, g_CaL = G_CAL;
    const double Ki = st[KI], Nai = st[NAI], Cai = st[CAI], Cass = st[CASS],
                 CaSR = st[CASR], Xr1 = st[XR1], Xr2 = st[XR2], Xs = st[XS],
                 m = st[M_], h = st[H_], j = st[J_], d = st[D_], f = st[F_],
                 f2 = st[F2_], fCass = st[FCASS], s = st[S_], r = st[R_],
                 Rp = st[RPRIME];

    const double E_Na = RTF * log(Nao / Nai);
    const double E_K = RTF * log(Ko / Ki);
    const double E_Ks = RTF * log((Ko + P_kna * Nao) / (Ki + P_kna * Nai));
    const double E_Ca = (RTF / 2.0) * log(Cao / Cai);

    double t1 = 1.0 / (1.0 + exp((-56.86 - V) / 9.03));
    const double m_inf = t1 * t1;
    const double alpha_m = 1.0 / (1.0 + exp((-60.0 - V) / 5.0));
    const double beta_m = 0.1 / (1.0 + exp((V + 35.0) / 5.0)) +
                          0.1 / (1.0 + exp((V - 50.0) / 200.0));
    const double tau_m = alpha_m * beta_m;

    t1 = 1.0 / (1.0 + exp((V + 71.55) / 7.43));
    const double h_inf = t1 * t1;
    double alpha_h, beta_h, alpha_j, beta_j;
    if (V < -40.0) {
        alpha_h = 0.057 * exp(-(V + 80.0) / 6.8);
        beta_h = 2.7 * exp(0.079 * V) + 3.1e5 * exp(0.3485 * V);
        alpha_j = ((-25428.0 * exp(0.2444 * V) - 6.948e-6 * exp(-0.04391 * V)) *
                   (V + 37.78)) / (1.0 + exp(0.311 * (V + 79.23)));
        beta_j = 0.02424 * exp(-0.01052 * V) / (1.0 + exp(-0.1378 * (V + 40.14)));
    } else {
        alpha_h = 0.0;
        beta_h = 0.77 / (0.13 * (1.0 + exp((V + 10.66) / -11.1)));
        alpha_j = 0.0;
        beta_j = 0.6 * exp(0.057 * V) / (1.0 + exp(-0.1 * (V + 32.0)));
    }
    const double tau_h = 1.0 / (alpha_h + beta_h + 1e-30);
    const double j_inf = h_inf;
    const double tau_j = 1.0 / (alpha_j + beta_j + 1e-30);
    const double i_Na = g_Na * m * m * m * h * j * (V - E_Na);

    const double xr1_inf = 1.0 / (1.0 + exp((-26.0 - V) / 7.0));
    const double tau_xr1 = 450.0 / (1.0 + exp((-45.0 - V) / 10.0)) * 6.0 /
                           (1.0 + exp((V + 30.0) / 11.5));
    const double xr2_inf = 1.0 / (1.0 + exp((V + 88.0) / 24.0));
    const double tau_xr2 = 3.0 / (1.0 + exp((-60.0 - V) / 20.0)) * 1.12 /
                           (1.0 + exp((V - 60.0) / 20.0));
    const double sqko = sqrt(Ko / 5.4);
    const double i_Kr = g_Kr * sqko * Xr1 * Xr2 * (V - E_K);

    const double xs_inf = 1.0 / (1.0 + exp((-5.0 - V) / 14.0));
    const double axs = 1400.0 / sqrt(1.0 + exp((5.0 - V) / 6.0));
    const double bxs = 1.0 / (1.0 + exp((V - 35.0) / 15.0));
    const double tau_xs = axs * bxs + 80.0;
    const double i_Ks = g_Ks * Xs * Xs * (V - E_Ks);

    const double ak1 = 0.1 / (1.0 + exp(0.06 * (V - E_K - 200.0)));
    const double bk1 = (3.0 * exp(2e-4 * (V - E_K + 100.0)) + exp(0.1 * (V - E_K - 10.0))) /
                       (1.0 + exp(-0.5 * (V - E_K)));
    const double xk1_inf = ak1 / (ak1 + bk1);
    const double i_K1 = g_K1 * sqko * xk1_inf * (V - E_K);

    double s_inf, tau_s;
    if (PH_ENDO_S[pheno]) {
        s_inf = 1.0 / (1.0 + exp((V + 28.0) / 5.0));
        tau_s = 1000.0 * exp(-(V + 67.0) * (V + 67.0) / 1000.0) + 8.0;
    } else {
        s_inf = 1.0 / (1.0 + exp((V + 20.0) / 5.0));
        tau_s = 85.0 * exp(-(V + 45.0) * (V + 45.0) / 320.0) +
                5.0 / (1.0 + exp((V - 20.0) / 5.0)) + 3.0;
    }
    const double r_inf = 1.0 / (1.0 + exp((20.0 - V) / 6.0));
    const double tau_r = 9.5 * exp(-(V + 40.0) * (V + 40.0) / 1800.0) + 0.8;
    const double i_to = g_to * r * s * (V - E_K);

    const double d_inf = 1.0 / (1.0 + exp((-8.0 - V) / 7.5));
    const double tau_d = (1.4 / (1.0 + exp((-35.0 - V) / 13.0)) + 0.25) * 1.4 /
                         (1.0 + exp((V + 5.0) / 5.0)) +
                         1.0 / (1.0 + exp((50.0 - V) / 20.0));
    const double f_inf = 1.0 / (1.0 + exp((V + 20.0) / 7.0));
    const double tau_f = 1102.5 * exp(-((V + 27.0) * (V + 27.0)) / 225.0) +
                         200.0 / (1.0 + exp((13.0 - V) / 10.0)) +
                         180.0 / (1.0 + exp((V + 30.0) / 10.0)) + 20.0;
    const double f2_inf = 0.67 / (1.0 + exp((V + 35.0) / 7.0)) + 0.33;
    const double tau_f2 = 562.0 * exp(-((V + 27.0) * (V + 27.0)) / 240.0) +
                          31.0 / (1.0 + exp((25.0 - V) / 10.0)) +
                          80.0 / (1.0 + exp((V + 30.0) / 10.0));
    const double cq = (Cass / 0.05) * (Cass / 0.05);
    const double fCass_inf = 0.6 / (1.0 + cq) + 0.4;
    const double tau_fCass = 80.0 / (1.0 + cq) + 2.0;

    const double exp2V = exp(2.0 * (V - 15.0) * FRT);
    double denom = exp2V - 1.0;
    if (fabs(denom) < 1e-10) denom = 1e-10;
    const double i_CaL = g_CaL * d * f * f2 * fCass * 4.0 * (V - 15.0) * F_c * F_c /
                         (Rgas * Tk) * (0.25 * Cass * exp2V - Cao) / denom;

    const double i_bNa = g_bna * (V - E_Na);
    const double i_bCa = g_bca * (V - E_Ca);
    const double i_pCa = g_pCa * Cai / (Cai + K_pCa);
    const double i_pK = g_pK * (V - E_K) / (1.0 + exp((25.0 - V) / 5.98));
    const double i_NaK = P_NaK * Ko / (Ko + K_mk) * Nai / (Nai + K_mNa) /
                         (1.0 + 0.1245 * exp(-0.1 * V * FRT) + 0.0353 * exp(-V * FRT));
    const double eVg = exp(gamma_ * V * FRT);
    const double eVgm1 = exp((gamma_ - 1.0) * V * FRT);
    const double i_NaCa = K_NaCa * (eVg * Nai * Nai * Nai * Cao - eVgm1 * Nao * Nao * Nao * Cai * alpha_) /
                          ((Km_Nai * Km_Nai * Km_Nai + Nao * Nao * Nao) * (Km_Ca + Cao) *
                           (1.0 + K_sat * eVgm1));

    const double I_ion = i_K1 + i_to + i_Kr + i_Ks + i_CaL + i_NaK + i_Na + i_bNa +
                         i_NaCa + i_bCa + i_pCa + i_pK;

    const double ecs = EC / CaSR;
    const double kcasr = max_sr - (max_sr - min_sr) / (1.0 + ecs * ecs);
    const double k1 = k1p / kcasr, k2 = k2p * kcasr;
    const double O = k1 * Cass * Cass * Rp / (k3 + k1 * Cass * Cass + 1e-30);
    const double i_rel = V_rel * O * (CaSR - Cass);
    const double i_up = Vmax_up / (1.0 + K_up * K_up / (Cai * Cai + 1e-30));
    const double i_leak = V_leak * (CaSR - Cai);
    const double i_xfer = V_xfer * (Cass - Cai);
    const double bufc = 1.0 / (1.0 + Buf_c * K_buf_c / ((Cai + K_buf_c) * (Cai + K_buf_c)));
    const double bufsr = 1.0 / (1.0 + Buf_sr * K_buf_sr / ((CaSR + K_buf_sr) * (CaSR + K_buf_sr)));
    const double bufss = 1.0 / (1.0 + Buf_ss * K_buf_ss / ((Cass + K_buf_ss) * (Cass + K_buf_ss)));

    const double dNai = -(i_Na + i_bNa + 3.0 * i_NaK + 3.0 * i_NaCa) * Cm_model / (V_c * F_c);
    const double dKi = -(i_K1 + i_to + i_Kr + i_Ks + i_pK - 2.0 * i_NaK) * Cm_model / (V_c * F_c);
    const double dCai = bufc * ((i_leak - i_up) * V_sr / V_c + i_xfer -
                                (i_bCa + i_pCa - 2.0 * i_NaCa) * Cm_model / (2.0 * V_c * F_c));
    const double dCaSR = bufsr * (i_up - i_rel - i_leak);
    const double dCass = bufss * (-i_CaL * Cm_model / (2.0 * V_ss * F_c) +
                                  i_rel * V_sr / V_ss - i_xfer * V_c / V_ss);

    st[M_] = rl(m, m_inf, tau_m, dt);
    st[H_] = rl(h, h_inf, tau_h, dt);
    st[J_] = rl(j, j_inf, tau_j, dt);
    st[XR1] = rl(Xr1, xr1_inf, tau_xr1, dt);
    st[XR2] = rl(Xr2, xr2_inf, tau_xr2, dt);
    st[XS] = rl(Xs, xs_inf, tau_xs, dt);
    st[D_] = rl(d, d_inf, tau_d, dt);
    st[F_] = rl(f, f_inf, tau_f, dt);
    st[F2_] = rl(f2, f2_inf, tau_f2, dt);
    st[FCASS] = rl(fCass, fCass_inf, tau_fCass, dt);
    st[S_] = rl(s, s_inf, tau_s, dt);
    st[R_] = rl(r, r_inf, tau_r, dt);
    st[RPRIME] = Rp + dt * (-k2 * Cass * Rp + k4 * (1.0 - Rp));
    st[NAI] = fmax(Nai + dt * dNai, 1e-3);
    st[KI] = fmax(Ki + dt * dKi, 1e-3);
    st[CAI] = fmax(Cai + dt * dCai, 1e-7);
    st[CASR] = fmax(CaSR + dt * dCaSR, 1e-7);
    st[CASS] = fmax(Cass + dt * dCass, 1e-7);
    return I_ion;
}

/* Vectorised over n cells: V (n), state (n x 18 row-major), pheno (n, 0..2),
 * optional per-cell g_Ks / g_Kr scales (NULL = 1).  Iion out (n). */
static int g_threads = 0;

int orc_num_threads(void) {
    if (g_threads > 0) return g_threads;
    const char *e = getenv("ORACLE_THREADS");
    long n = e ? atol(e) : sysconf(_SC_NPROCESSORS_ONLN);
    if (n < 1) n = 1;
    if (n > 256) n = 256;
    g_threads = (int)n;
    return g_threads;
}

void orc_set_threads(int n) { g_threads = n < 1 ? 1 : n; }

typedef struct {
    int64_t n; const double *V; double *state; double dt; const int8_t *pheno;
    const double *gks_s, *gkr_s; double *Iion; int nt;
} step_ctx;
typedef struct { step_ctx *c; int tid; } step_arg;

static void *step_worker(void *p) {
    step_arg *a = (step_arg *)p;
    step_ctx *c = a->c;
    int64_t lo = c->n * a->tid / c->nt, hi = c->n * (a->tid + 1) / c->nt;
    for (int64_t i = lo; i < hi; ++i)
        c->Iion[i] = orc_ttp06_cell(c->V[i], c->state + i * NSTATE, c->dt, c->pheno[i],
                                    c->gks_s ? c->gks_s[i] : 1.0, c->gkr_s ? c->gkr_s[i] : 1.0);
    return NULL;
}

/* Vectorised over n cells: V (n), state (n x 18 row-major), pheno (n, 0..2),
 * optional per-cell g_Ks / g_Kr scales (NULL = 1).  Iion out (n). */
void orc_ttp06_step(int64_t n, const double *V, double *state, double dt,
                    const int8_t *pheno, const double *gks_s, const double *gkr_s,
                    double *Iion) {
    int nt = orc_num_threads();
    if (n < 4096) nt = 1;
    step_ctx c = {n, V, state, dt, pheno, gks_s, gkr_s, Iion, nt};
    pthread_t th[256];
    step_arg args[256];
    for (int t = 0; t < nt; ++t) {
        args[t].c = &c; args[t].tid = t;
        if (t) pthread_create(&th[t], NULL, step_worker, &args[t]);
    }
    step_worker(&args[0]);
    for (int t = 1; t < nt; ++t) pthread_join(th[t], NULL);
}

/*
 * Explicit (theta = 0) monodomain time loop over the assembled global
 * Laplacian L (CSR, FP64, rows already divided by the membrane loading).
 * N nodes in reference order [Purkinje | myocardium]; pheno per node.
 * Stimulus: n_sites sites, each a node list (CSR site_ptr/site_nodes) with
 * amplitude site_amp [uA/mm^2]; site_on[step * n_sites + s] = 1 when the
 * site fires at t = step * dt (the host evaluates the reference's
 * _stim_active).  Within a site a node counts once; sites add.
 * After every step the myocardial part V[n_skip:] is written to
 * snaps[(step / snap_every)] when step % snap_every == 0 (float32), which is
 * the reference's vm snapshot (labelled t = step * dt).  Optionally the
 * Purkinje part V[:n_skip] likewise into psnaps.
 * V (N) and state (N x 18) are advanced in place.  Returns 0.
 */
typedef struct {
    int64_t N, n_skip;
    const int64_t *L_ptr; const int32_t *L_idx; const double *L_val;
    const int8_t *pheno; const double *gks_s, *gkr_s;
    double dt, Cm; int64_t n_steps;
    int n_sites; const int64_t *site_ptr; const int32_t *site_nodes;
    const double *site_amp; const uint8_t *site_on;
    double *V, *state; int64_t snap_every; float *snaps, *psnaps;
    double *Istim, *Vs; unsigned char *mark;
    int nt; pthread_barrier_t bar;
} run_ctx;
typedef struct { run_ctx *c; int tid; } run_arg;

static void *run_worker(void *p) {
    run_arg *a = (run_arg *)p;
    run_ctx *c = a->c;
    const int64_t N = c->N;
    const int64_t lo = N * a->tid / c->nt, hi = N * (a->tid + 1) / c->nt;
    int64_t snap_i = 0;
    for (int64_t step = 0; step < c->n_steps; ++step) {
        if (a->tid == 0) {
            /* stimulus: sum of amp * mask over firing sites (a node counts
             * once per site, sites add) */
            memset(c->Istim, 0, sizeof(double) * N);
            for (int s = 0; s < c->n_sites; ++s) {
                if (!c->site_on[step * c->n_sites + s]) continue;
                for (int64_t q = c->site_ptr[s]; q < c->site_ptr[s + 1]; ++q) c->mark[c->site_nodes[q]] = 1;
                for (int64_t q = c->site_ptr[s]; q < c->site_ptr[s + 1]; ++q) {
                    int32_t nd = c->site_nodes[q];
                    if (c->mark[nd]) { c->Istim[nd] += c->site_amp[s]; c->mark[nd] = 0; }
                }
            }
        }
        pthread_barrier_wait(&c->bar);
        for (int64_t i = lo; i < hi; ++i) {
            double ii = orc_ttp06_cell(c->V[i], c->state + i * NSTATE, c->dt, c->pheno[i],
                                       c->gks_s ? c->gks_s[i] : 1.0, c->gkr_s ? c->gkr_s[i] : 1.0);
            double Iion_pde = ii * c->Cm;
            c->Vs[i] = c->V[i] + (c->dt / c->Cm) * (-Iion_pde + c->Istim[i]);
        }
        pthread_barrier_wait(&c->bar);
        for (int64_t i = lo; i < hi; ++i) {
            double acc = 0.0;
            for (int64_t q = c->L_ptr[i]; q < c->L_ptr[i + 1]; ++q) acc += c->L_val[q] * c->Vs[c->L_idx[q]];
            double v = c->Vs[i] + (c->dt / c->Cm) * acc;
            c->V[i] = v < -150.0 ? -150.0 : (v > 80.0 ? 80.0 : v);
        }
        pthread_barrier_wait(&c->bar);
        if (c->snap_every > 0 && step % c->snap_every == 0) {
            if (c->snaps) {
                float *dst = c->snaps + snap_i * (N - c->n_skip);
                for (int64_t i = (lo > c->n_skip ? lo : c->n_skip); i < hi; ++i)
                    dst[i - c->n_skip] = (float)c->V[i];
            }
            if (c->psnaps) {
                float *dst = c->psnaps + snap_i * c->n_skip;
                for (int64_t i = lo; i < hi && i < c->n_skip; ++i) dst[i] = (float)c->V[i];
            }
            ++snap_i;
        }
    }
    return NULL;
}

/*
 * Explicit (theta = 0) monodomain time loop over the assembled global
 * Laplacian L (CSR, FP64, rows already divided by the membrane loading).
 * N nodes in reference order [Purkinje | myocardium]; pheno per node.
 * Stimulus: n_sites sites, each a node list (CSR site_ptr/site_nodes) with
 * amplitude site_amp [uA/mm^2]; site_on[step * n_sites + s] = 1 when the
 * site fires at t = step * dt (the host evaluates the reference's
 * _stim_active).  After every step the myocardial part V[n_skip:] is written
 * to snaps[step / snap_every] when step % snap_every == 0 (float32): the
 * reference's vm snapshot, labelled t = step * dt.  Optionally the Purkinje
 * part V[:n_skip] likewise into psnaps.  V (N) and state (N x 18) are
 * advanced in place.  Returns 0, or -2 when out of host memory.
 */
int orc_mono_run(int64_t N, int64_t n_skip,
                 const int64_t *L_ptr, const int32_t *L_idx, const double *L_val,
                 const int8_t *pheno, const double *gks_s, const double *gkr_s,
                 double dt, double Cm, int64_t n_steps,
                 int n_sites, const int64_t *site_ptr, const int32_t *site_nodes,
                 const double *site_amp, const uint8_t *site_on,
                 double *V, double *state,
                 int64_t snap_every, float *snaps, float *psnaps) {
    run_ctx c;
    memset(&c, 0, sizeof(c));
    c.N = N; c.n_skip = n_skip; c.L_ptr = L_ptr; c.L_idx = L_idx; c.L_val = L_val;
    c.pheno = pheno; c.gks_s = gks_s; c.gkr_s = gkr_s; c.dt = dt; c.Cm = Cm;
    c.n_steps = n_steps; c.n_sites = n_sites; c.site_ptr = site_ptr;
    c.site_nodes = site_nodes; c.site_amp = site_amp; c.site_on = site_on;
    c.V = V; c.state = state; c.snap_every = snap_every; c.snaps = snaps; c.psnaps = psnaps;
    c.Istim = (double *)calloc(N, sizeof(double));
    c.Vs = (double *)malloc(sizeof(double) * N);
    c.mark = (unsigned char *)calloc(N, 1);
    if (!c.Istim || !c.Vs || !c.mark) { free(c.Istim); free(c.Vs); free(c.mark); return -2; }
    int nt = orc_num_threads();
    if (N < 4096) nt = 1;
    c.nt = nt;
    pthread_barrier_init(&c.bar, NULL, nt);
    pthread_t th[256];
    run_arg args[256];
    for (int t = 0; t < nt; ++t) {
        args[t].c = &c; args[t].tid = t;
        if (t) pthread_create(&th[t], NULL, run_worker, &args[t]);
    }
    run_worker(&args[0]);
    for (int t = 1; t < nt; ++t) pthread_join(th[t], NULL);
    pthread_barrier_destroy(&c.bar);
    free(c.Istim); free(c.Vs); free(c.mark);
    return 0;
}

/*
 * Theta-scheme (Crank-Nicolson at theta = 0.5) monodomain time loop: the
 * reference's default diffusion half (pipeline.py:1383-1391, anisotropic
 * solver :1784-1790).  Per step: ionic step on V^n, V* as orc_mono_run, then
 * A V^{n+1} = b with A = (Cm/dt) I - theta L, b = (Cm/dt) V* + (1 - theta)
 * L V*, solved by the reference's Jacobi-preconditioned BiCGSTAB from x0 = V*
 * (_build_cn_matrix pipeline.py:662-688, _bicgstab :691-754, restated
 * below step by step), clamped to [-150, 80].  Serial.  iters (may be NULL)
 * receives the BiCGSTAB iteration count summed over the steps.
 */
static void cn_apply(int64_t N, const int64_t *Lp, const int32_t *Li, const double *Lv,
                     double scale, double theta, const double *x, double *y) {
    for (int64_t i = 0; i < N; ++i) {
        double acc = 0.0;
        for (int64_t q = Lp[i]; q < Lp[i + 1]; ++q) acc += Lv[q] * x[Li[q]];
        y[i] = scale * x[i] - theta * acc;
    }
}
static double dotv(int64_t N, const double *a, const double *b) {
    double s = 0.0;
    for (int64_t i = 0; i < N; ++i) s += a[i] * b[i];
    return s;
}

/* _bicgstab (pipeline.py:691-754); x holds x0 on entry.  Returns iterations. */
static int64_t cn_bicgstab(int64_t N, const int64_t *Lp, const int32_t *Li, const double *Lv,
                           double scale, double theta, const double *Minv, const double *b,
                           double *x, double tol, int64_t maxiter, double *w) {
    double *r = w, *rh = w + N, *v = w + 2 * N, *p = w + 3 * N, *ph = w + 4 * N,
           *s = w + 5 * N, *sh = w + 6 * N, *t = w + 7 * N;
    cn_apply(N, Lp, Li, Lv, scale, theta, x, t);
    for (int64_t i = 0; i < N; ++i) { r[i] = b[i] - t[i]; rh[i] = r[i]; v[i] = 0.0; p[i] = 0.0; }
    double rho_prev = 1.0, alpha = 1.0, omega = 1.0;
    const double b_norm = sqrt(dotv(N, b, b));
    if (b_norm == 0.0) return 0;
    int64_t it = 0;
    for (; it < maxiter; ++it) {
        double rho = dotv(N, rh, r);
        if (fabs(rho) < 1e-300) {
            for (int64_t i = 0; i < N; ++i) rh[i] = r[i];
            rho = dotv(N, rh, r);
        }
        if (it == 0) {
            for (int64_t i = 0; i < N; ++i) p[i] = r[i];
        } else {
            const double beta = (rho / rho_prev) * (alpha / omega);
            for (int64_t i = 0; i < N; ++i) p[i] = r[i] + beta * (p[i] - omega * v[i]);
        }
        for (int64_t i = 0; i < N; ++i) ph[i] = Minv[i] * p[i];
        cn_apply(N, Lp, Li, Lv, scale, theta, ph, v);
        const double da = dotv(N, rh, v);
        if (fabs(da) < 1e-300) break;
        alpha = rho / da;
        for (int64_t i = 0; i < N; ++i) s[i] = r[i] - alpha * v[i];
        if (sqrt(dotv(N, s, s)) < tol * b_norm) {
            for (int64_t i = 0; i < N; ++i) x[i] += alpha * ph[i];
            ++it;
            break;
        }
        for (int64_t i = 0; i < N; ++i) sh[i] = Minv[i] * s[i];
        cn_apply(N, Lp, Li, Lv, scale, theta, sh, t);
        const double dw = dotv(N, t, t);
        omega = fabs(dw) > 1e-300 ? dotv(N, t, s) / dw : 0.0;
        for (int64_t i = 0; i < N; ++i) {
            x[i] += alpha * ph[i] + omega * sh[i];
            r[i] = s[i] - omega * t[i];
        }
        rho_prev = rho;
        if (sqrt(dotv(N, r, r)) / b_norm < tol) { ++it; break; }
        if (fabs(omega) < 1e-300) { ++it; break; }
    }
    return it;
}

int orc_mono_run_cn(int64_t N, int64_t n_skip,
                    const int64_t *L_ptr, const int32_t *L_idx, const double *L_val,
                    const int8_t *pheno, const double *gks_s, const double *gkr_s,
                    double dt, double Cm, int64_t n_steps,
                    int n_sites, const int64_t *site_ptr, const int32_t *site_nodes,
                    const double *site_amp, const uint8_t *site_on,
                    double *V, double *state,
                    int64_t snap_every, float *snaps, float *psnaps,
                    double theta, double tol, int64_t maxiter, int64_t *iters) {
    const double scale = Cm / dt;
    double *Istim = (double *)calloc(N, sizeof(double));
    double *Vs = (double *)malloc(sizeof(double) * N);
    double *b = (double *)malloc(sizeof(double) * N);
    double *Minv = (double *)malloc(sizeof(double) * N);
    double *w = (double *)malloc(sizeof(double) * 8 * N);
    unsigned char *mark = (unsigned char *)calloc(N, 1);
    if (!Istim || !Vs || !b || !Minv || !w || !mark) {
        free(Istim); free(Vs); free(b); free(Minv); free(w); free(mark);
        return -2;
    }
    /* M_inv = 1 / (scale - theta diag L), pipeline.py:686-687 */
    for (int64_t i = 0; i < N; ++i) {
        double dl = 0.0;
        for (int64_t q = L_ptr[i]; q < L_ptr[i + 1]; ++q)
            if (L_idx[q] == i) dl += L_val[q];
        double da = scale - theta * dl;
        Minv[i] = 1.0 / (da > 1e-30 ? da : 1e-30);
    }
    int64_t snap_i = 0, it_sum = 0;
    for (int64_t step = 0; step < n_steps; ++step) {
        memset(Istim, 0, sizeof(double) * N);
        for (int s = 0; s < n_sites; ++s) {
            if (!site_on[step * n_sites + s]) continue;
            for (int64_t q = site_ptr[s]; q < site_ptr[s + 1]; ++q) mark[site_nodes[q]] = 1;
            for (int64_t q = site_ptr[s]; q < site_ptr[s + 1]; ++q) {
                int32_t nd = site_nodes[q];
                if (mark[nd]) { Istim[nd] += site_amp[s]; mark[nd] = 0; }
            }
        }
        for (int64_t i = 0; i < N; ++i) {
            double ii = orc_ttp06_cell(V[i], state + i * NSTATE, dt, pheno[i],
                                       gks_s ? gks_s[i] : 1.0, gkr_s ? gkr_s[i] : 1.0);
            Vs[i] = V[i] + (dt / Cm) * (-(ii * Cm) + Istim[i]);
        }
        for (int64_t i = 0; i < N; ++i) {
            double acc = 0.0;
            for (int64_t q = L_ptr[i]; q < L_ptr[i + 1]; ++q) acc += L_val[q] * Vs[L_idx[q]];
            b[i] = scale * Vs[i] + (1.0 - theta) * acc;
        }
        memcpy(V, Vs, sizeof(double) * N);
        it_sum += cn_bicgstab(N, L_ptr, L_idx, L_val, scale, theta, Minv, b, V, tol, maxiter, w);
        for (int64_t i = 0; i < N; ++i) V[i] = V[i] < -150.0 ? -150.0 : (V[i] > 80.0 ? 80.0 : V[i]);
        if (snap_every > 0 && step % snap_every == 0) {
            if (snaps)
                for (int64_t i = n_skip; i < N; ++i) snaps[snap_i * (N - n_skip) + i - n_skip] = (float)V[i];
            if (psnaps)
                for (int64_t i = 0; i < n_skip; ++i) psnaps[snap_i * n_skip + i] = (float)V[i];
            ++snap_i;
        }
    }
    if (iters) *iters = it_sum;
    free(Istim); free(Vs); free(b); free(Minv); free(w); free(mark);
    return 0;
}
