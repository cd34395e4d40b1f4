/*
 * hrdaya_b200.h -- C ABI of the B200-native HrdayaPy hot path.
 *
 * One shared library (libhrdaya_b200.so) exports these entry points.  They
 * take plain pointers and sizes; device buffers are owned by the handles
 * (allocated at create, freed at destroy) and results are copied out to
 * caller-owned memory, host or device.  Every call returns an hp_status;
 * hp_last_error() gives the message of the last failure on this thread.
 * Handles are not thread-safe (same contract as the reference's solvers,
 * which are single-threaded Python).  `stream` arguments are cudaStream_t
 * passed as void* (NULL = legacy default stream).
 *
 * Reference interfaces replaced (paths inside the HrdayaPy project):
 *   hp_mono_*   -- the time loop of run_coupled
 *                  (simulation/functions/purkinje_myocardium_pipeline.py:1030-1463)
 *                  and purkinje_myocardium_anisotropic_solver
 *                  (anisotropic_simulation/functions/
 *                   purkinje_myocardium_anisotropic_solver.py:1308-1881):
 *                  HeteroIonicSolver.step (ionic_models/hetero_solver.py:141-194),
 *                  the V update (pipeline.py:1379-1382), the global
 *                  Laplacian mat-vec and solve (pipeline.py:578-754), the clamp,
 *                  the Vm snapshot / animation frame writers (pipeline.py:1395-1412)
 *                  and the activation-time extraction of
 *                  compute_activation_maps (activation_maps.py:295-350).
 *   hp_torso_*  -- make_gpu_solver / solve_frame / _pcg_gpu
 *                  (ecg/functions/compute_bspm.py:164-436) over the stiffness
 *                  operator of _assemble_stiffness (ecg/functions/build_torso_grid.py:276-397).
 */
#ifndef HRDAYA_B200_H
#define HRDAYA_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  HP_OK = 0,
  HP_ERR_INVALID = 1,       /* bad argument (maps to ValueError) */
  HP_ERR_OOM = 2,           /* device allocation failed */
  HP_ERR_CUDA = 3,          /* CUDA runtime error */
  HP_ERR_NOT_CONVERGED = 4, /* iteration limit reached */
  HP_ERR_STAGNATED = 5,     /* Krylov stagnation / breakdown */
  HP_ERR_NONFINITE = 6,     /* NaN / Inf detected */
  HP_ERR_TIMEOUT = 7,       /* bounded device wait expired */
  HP_ERR_UNSUPPORTED = 8    /* configuration not built into this library */
} hp_status;

/* Message of the last failing call on this thread ("" if none). */
const char *hp_last_error(void);
/* Library version string. */
const char *hp_version(void);

/* ------------------------------------------------------------------ */
/* Monodomain (fused TTP06 + 19-point stencil + activation recording)  */
/* ------------------------------------------------------------------ */

/* Voxel tag bits (uint32 per voxel slot). */
#define HP_TAG_PHENO_MASK 0x3u        /* 0 = not tissue, 1 endo, 2 mid, 3 epi */
#define HP_TAG_FACE_SHIFT 2           /* 6 bits: +i -i +j -j +k -k neighbour in mask */
#define HP_TAG_DIAG_SHIFT 8           /* 12 bits: edge-diagonal neighbours in mask */
#define HP_TAG_STIM_SHIFT 20          /* 8 bits: stimulus-site membership */
#define HP_TAG_PMJ (1u << 28)         /* voxel coupled to Purkinje junction(s) */
#define HP_TAG_SURF (1u << 29)        /* voxel is an animation-surface node */
#define HP_MAX_SITES 8
#define HP_MAX_VARIANTS 64

/*
 * Geometry and parameters of one monodomain problem (or of a batched
 * ensemble of independent variants, concatenated brick by brick).
 * All pointers are HOST pointers; hp_mono_create copies them to the device.
 *
 * Voxels live in bricks of bi x bj x bk (k fastest); slot = brick * bv +
 * (li * bj + lj) * bk + lk.  brick_nbr holds, per brick, the 27 neighbouring
 * brick ids in (di, dj, dk) order with di slowest, -1 where absent (index 13
 * is the brick itself).
 *
 * Diffusion coefficients are pre-scaled by dt / (Cm * Ai) so that one
 * explicit step is V += sum_j coef_ij (V_j - V_i):
 *   isotropic:   coef = iso_coef for every face neighbour in the mask;
 *   anisotropic: face coef to +i/+j/+k stored per voxel (wface, 3 x n_slots,
 *                zero where the edge does not exist), edge-diagonal coef
 *                = +/-(doff_a + doff_b) / 4 from the per-voxel off-diagonal
 *                tensor components doff (3 x n_slots: D01, D02, D12 scaled).
 */
typedef struct {
  int32_t n_bricks;
  int32_t bi, bj, bk;           /* brick shape; must be a compiled shape */
  int32_t anisotropic;          /* 0: 7-point, 1: 19-point */
  const int32_t *brick_nbr;     /* n_bricks x 27 */
  const uint32_t *tag;          /* n_slots */
  const float *wface;           /* 3 x n_slots (anisotropic) */
  const float *doff;            /* 3 x n_slots (anisotropic) */
  float iso_coef;               /* isotropic face coefficient */
  const uint8_t *brick_variant; /* n_bricks, or NULL (all variant 0) */
  int32_t n_variants;
  const float *variant_gks;     /* n_variants multipliers of g_Ks */
  const float *variant_gkr;     /* n_variants multipliers of g_Kr */

  /* Purkinje network: n_pk nodes, CSR neighbours; a neighbour index
   * j >= 0 is a Purkinje node, j < 0 is myocardial slot (-j - 1). */
  int32_t n_pk;
  const int32_t *pk_ptr;        /* n_pk + 1 */
  const int32_t *pk_idx;
  const float *pk_coef;
  const uint8_t *pk_stim;       /* n_pk stimulus-site bits */
  const uint8_t *pk_variant;    /* n_pk, or NULL */
  /* myocardial side of the junctions: for voxels tagged HP_TAG_PMJ,
   * pmj_row[slot] indexes the CSR (pmj_ptr, pmj_pk, pmj_coef). */
  int32_t n_pmj_rows;
  const int32_t *pmj_row;       /* n_slots (only read where tagged) */
  const int32_t *pmj_ptr;       /* n_pmj_rows + 1 */
  const int32_t *pmj_pk;
  const float *pmj_coef;

  /* time stepping and stimulus (each variant has its own n_sites sites) */
  double dt;                    /* ms */
  double Cm;                    /* uF/mm^2 */
  float v0;                     /* initial membrane potential, mV */
  int64_t n_steps;              /* total steps of the run */
  int32_t n_sites;
  const float *site_amp;        /* n_variants x n_sites, uA/mm^2 */
  const uint8_t *site_on;       /* n_variants x (n_steps + 1) bitmasks: sites firing at t = step * dt */

  /* outputs */
  int32_t n_myo;                /* myocardial nodes in reference order */
  const int32_t *slot_of_node;  /* n_myo */
  int64_t vm_every;             /* Vm snapshot every vm_every steps (0 = off) */
  int32_t n_surf;               /* animation surface nodes */
  const int32_t *surf_of_slot;  /* n_slots (read where HP_TAG_SURF) */
  int64_t frame_every;          /* animation frame every frame_every steps (0 = off) */
  float act_threshold;          /* mV, upstroke crossing */
  float deact_threshold;        /* mV, downstroke crossing */
  int32_t max_events;           /* activation events kept per voxel (1..16) */

  /* step kernel (all give bit-identical results): HP_MONO_KERNEL_AUTO is
   * the split step, the fastest on B200 for every compiled brick shape */
  int32_t kernel;

  /* diffusion half: theta = 0 is the explicit update above; 0 < theta <= 1
   * solves (I - theta Lh) V_{i+1} = W_i + (1 - theta) Lh W_i each step by
   * Jacobi-preconditioned CG from V_{i+1} = W_i (reference: BiCGSTAB on the
   * same system, pipeline.py:662-754 and :1383-1391), stopping when
   * ||r|| <= cn_tol ||rhs|| (cn_tol below 1e-7 is raised to 1e-7, FP32
   * vectors) or after cn_max_iter iterations.  pk_weight = Ai_P / Ai_M, the
   * Purkinje over the tissue membrane loading (the inner product that makes
   * the operator symmetric).  Needs the split step (kernel AUTO or SPLIT);
   * CUDA-graph chunks are not used (the host tests convergence). */
  double theta;
  double cn_tol;
  int32_t cn_max_iter;
  float pk_weight;
} HpMonoDesc;

#define HP_MONO_KERNEL_AUTO 0
#define HP_MONO_KERNEL_BRICK 1     /* one CTA per brick, plain halo loads */
#define HP_MONO_KERNEL_PIPELINED 2 /* persistent CTAs, cp.async double-buffered bricks */
#define HP_MONO_KERNEL_SPLIT 3     /* diffusion launch per brick + ionic launch per tissue slot */

typedef struct HpMono HpMono;

/* Allocates device state, uploads the description, initialises every cell to
 * the TTP06 resting state at v0 and runs the ionic half-step of step 0.  The
 * returned handle is bound to the current device. */
hp_status hp_mono_create(const HpMonoDesc *desc, HpMono **out, void *stream);
/* Advances n steps (n <= remaining).  Kernels are enqueued on `stream`; time
 * loops of `graph_chunk` > 0 steps are replayed from a CUDA graph. */
hp_status hp_mono_run(HpMono *h, int64_t n, int32_t graph_chunk, void *stream);
/* Steps done so far. */
int64_t hp_mono_steps_done(const HpMono *h);
/* Theta-scheme solver counters since creation: CG iterations, solves (one
 * per step), solves stopped by cn_max_iter, and breakdowns (<p, Ap> <= 0).
 * All zero at theta = 0.  Any output may be NULL; synchronises the device. */
hp_status hp_mono_cn_stats(HpMono *h, int64_t *iterations, int64_t *solves,
                           int64_t *unconverged, int64_t *breakdowns);
/* Step kernel in use (HP_MONO_KERNEL_BRICK, _PIPELINED or _SPLIT), its grid size
 * and dynamic shared memory per CTA; any output may be NULL. */
hp_status hp_mono_kernel_info(const HpMono *h, int32_t *kernel, int32_t *grid, int64_t *smem_bytes);
/* Copies snapshots [f0, f0 + nf) (each n_myo floats, reference node order)
 * to dst; dst_on_device selects cudaMemcpyDeviceToDevice. */
hp_status hp_mono_copy_vm(HpMono *h, int64_t f0, int64_t nf, float *dst,
                          int32_t dst_on_device, void *stream);
/* Animation frames [f0, f0 + nf): surface part (n_surf floats each) and
 * Purkinje part (n_pk floats each); either destination may be NULL. */
hp_status hp_mono_copy_frames(HpMono *h, int64_t f0, int64_t nf, float *dst_surf,
                              float *dst_pk, int32_t dst_on_device, void *stream);
/* Activation / deactivation events in reference node order:
 * act (max_events x n_myo, NaN = none), n_act (n_myo); same for deact.
 * Host destinations. */
hp_status hp_mono_copy_events(HpMono *h, float *act, int32_t *n_act, float *deact,
                              int32_t *n_deact, void *stream);
/* Current membrane potential after the last step: myocardium (n_myo, node
 * order) and Purkinje (n_pk).  Host destinations, either may be NULL. */
hp_status hp_mono_copy_v(HpMono *h, float *v_myo, float *v_pk, void *stream);
/* Raw state access for checkpointing: the 18 TTP06 variables of every slot
 * (18 x n_slots) and Purkinje node (18 x n_pk) as last written. */
hp_status hp_mono_copy_state(HpMono *h, float *state_slots, float *state_pk, void *stream);
/* Halo exchange of a heart split into slabs over several handles (one per
 * GPU; hrdayapy_b200.slab): the post-ionic potential W that the next step's
 * diffusion half reads, at n slots listed in device memory.  gather copies
 * W[slots[q]] to out[q], scatter writes in[q] to W[slots[q]] (device
 * buffers, both on `stream`).  No counterpart in the reference, which runs
 * one heart on one device (pipeline.py:1347-1420). */
hp_status hp_mono_w_gather(HpMono *h, const int32_t *slots, int64_t n, float *out, void *stream);
hp_status hp_mono_w_scatter(HpMono *h, const int32_t *slots, int64_t n, const float *in,
                            void *stream);
hp_status hp_mono_destroy(HpMono *h);

/* ------------------------------------------------------------------ */
/* Torso forward solve (per-frame Poisson, Jacobi-PCG)                 */
/* ------------------------------------------------------------------ */

#define HP_MAX_MATERIALS 16

/* Stopping rule of a frame solve. */
typedef enum {
  HP_STOP_REL = 0,   /* FP64 true residual ||b - A x|| / ||b|| <= tol */
  HP_STOP_RMS = 1,   /* sqrt(mean(z^2)) < tol (z = M^-1 r, volts), reference 'rms' */
  HP_STOP_LINF = 2,  /* max |z| < tol, reference 'linf' */
  HP_STOP_P99 = 3    /* 0.99 quantile of |z| (linear interpolation) < tol, reference 'p99' */
} hp_stop_rule;

/*
 * Torso grid and heart source geometry.  HOST pointers, copied at create.
 *
 * The torso is a dense grid ni x nj x nk (k fastest) of material labels;
 * conductivity sigma[label] in S/m (label 0 = air, sigma 0).  A voxel is an
 * unknown when its label is not 0 ("active"); rows are numbered in flat
 * (i, j, k) order of the active voxels, as the reference's active_ids.  Face
 * conductance = harmonic mean of the two sigmas / h^2, air faces Neumann.
 * pin_row is fixed to 0 (reference potential).
 *
 * Heart: n_heart fine voxels with their 6 face neighbours (heart_nbr,
 * n_heart x 6, -1 = none) for the source Laplacian, and the coarse row each
 * voxel projects to (proj, -1 = outside the torso).  Per frame:
 *   src_i = coeff * (K Vm * 1e-3)_i - mean over projected voxels,
 *   b_row = sum_{i -> row} src_i / n_expected,  b[pin_row] = 0.
 */
typedef struct {
  int32_t ni, nj, nk;
  double h_m;                   /* torso voxel size, metres */
  const uint8_t *label;         /* ni * nj * nk */
  int32_t n_materials;
  const double *sigma;          /* n_materials, S/m */
  int64_t pin_row;              /* row index of the pinned node */
  int32_t n_heart;
  const int32_t *heart_nbr;     /* n_heart x 6 */
  const int32_t *proj;          /* n_heart, coarse row or -1 */
  double coeff;                 /* sigma_i / h_fine^2 */
  double n_expected;            /* fine voxels per coarse voxel */
  int32_t n_read;               /* read-out rows (surface nodes, electrodes) */
  const int64_t *read_rows;     /* n_read */
  /* Smoothed boundary method (build_torso_grid.py:130-186, :276-386;
   * compute_bspm.py:413-414): NULL for the sharp boundary, else the domain
   * function psi (ni * nj * nk, > 0 exactly where label != 0).  Every face
   * conductance is multiplied by the harmonic mean 2 psi_k psi_n /
   * (psi_k + psi_n) and the right-hand side by psi.  Jacobi-PCG only: the
   * flexible-CG preconditioners refuse such a handle. */
  const float *psi;
} HpTorsoDesc;

typedef struct {
  int32_t iterations;           /* CG iterations of the last frame */
  int32_t status;               /* hp_status of the last frame */
  double rel_residual;          /* FP64 true ||b - A x|| / ||b|| at exit */
  double stat;                  /* value of the chosen stopping statistic */
  int32_t restarts;             /* residual replacements */
} HpSolveStats;

typedef struct HpTorso HpTorso;

hp_status hp_torso_create(const HpTorsoDesc *desc, HpTorso **out, void *stream);
/* Number of active rows (unknowns). */
int64_t hp_torso_rows(const HpTorso *h);
/* Solves one frame: vm (n_heart floats, mV) is read from host or device
 * memory (vm_on_device); warm start from the previous frame's solution
 * (zero for the first).  Writes the read-out potentials (n_read floats, mV)
 * to out (host or device, out_on_device).  tol/rule select the stopping
 * rule; max_iter bounds the iterations. */
hp_status hp_torso_solve_frame(HpTorso *h, const float *vm, int32_t vm_on_device, float *out,
                               int32_t out_on_device, double tol, int32_t rule,
                               int32_t max_iter, HpSolveStats *stats, void *stream);
/* Copies the full potential field (rows, FP64 volts) of the last frame to
 * host memory. */
hp_status hp_torso_copy_solution(HpTorso *h, double *x_rows, void *stream);
/* Copies the right-hand side (rows, FP32) of the last frame to host memory. */
hp_status hp_torso_copy_rhs(HpTorso *h, float *b_rows, void *stream);
/* Forgets the warm start (next frame starts from zero). */
hp_status hp_torso_reset(HpTorso *h);
hp_status hp_torso_destroy(HpTorso *h);

/*
 * Allocation-free FP64 true-residual check (no counterpart in the reference).
 * For callers that may not allocate device memory (a host framework that
 * owns every allocation, a real-time loop, a fixed memory budget): computes
 * out[0] = ||b - A x|| and out[1] = ||b|| (host doubles) for the torso
 * operator of hp_torso_create, with no cudaMalloc -- its only scratch is a
 * fixed array inside the library of (4 + 2 * HP_NOALLOC_MAX_BLOCKS) doubles
 * (1,048,608 bytes, about 1.0 MiB, per GPU, held until exit).  label
 * (uint8), x (fp64) and b (fp32) are device arrays over the PADDED grid
 * (ni+2) x (nj+2) x (nk+2), k fastest, whose one-voxel border must be air
 * (a nonzero border label is rejected with HP_ERR_INVALID); pin_cell is the
 * padded flat index of the pinned voxel (-1: none); sigma (host) holds
 * n_materials conductivities in S/m (label 0 = air).  Padded grids above
 * HP_NOALLOC_MAX_CELLS are rejected with HP_ERR_INVALID.  The call is
 * synchronous (it waits for its stream before returning).  Every call
 * shares the scratch array: calls that overlap on the GPU race.  The first
 * call on a device resolves the array's address on that device and keeps
 * it, so make it before any stream capture, and do not use the entry point
 * across a cudaDeviceReset.
 */
#define HP_NOALLOC_MAX_BLOCKS 65536
#define HP_NOALLOC_MAX_CELLS (HP_NOALLOC_MAX_BLOCKS * 256LL)
hp_status hp_torso_residual_noalloc(int32_t ni, int32_t nj, int32_t nk, const uint8_t *label,
                                    const double *sigma, int32_t n_materials, double h_m,
                                    int64_t pin_cell, const double *x, const float *b,
                                    double *out, void *stream);

/* ------------------------------------------------------------------ */
/* Learned preconditioner building block: tcgen05 3x3x3 convolution    */
/* ------------------------------------------------------------------ */

/*
 * One 3x3x3 convolution with zero padding 1 on the 5th-generation tensor
 * cores (no counterpart in the reference, which has no learned part).
 * X: device bf16 [D][H][W][cin]; Wp: device bf16 weights packed
 * [27][cin/8][cout][8] (tap = 9 kz + 3 ky + kx, see hrdayapy_b200/convref.py);
 * bias: device fp32 [cout]; Y: device bf16 [D][H][W][cout], or fp32
 * [D][H][W] for epi = 3.  epi: 0 relu(acc + bias), 1 acc + bias,
 * 2 acc * (mask > 0) (mask: bf16 [D][H][W][cout]), 3 acc[:, 0] + bias[0].
 * W must be a multiple of 128; cin / cout among the compiled pairs.
 * *err (device int) receives nonzero if a bounded device wait expired.
 */
hp_status hp_conv3_forward(const void *X, const void *Wp, const float *bias, void *Y,
                           const void *mask, int32_t D, int32_t H, int32_t W, int32_t cin,
                           int32_t cout, int32_t epi, int32_t *err, void *stream);

/*
 * Weight and bias gradients of one 3x3x3 convolution (zero padding 1) on the
 * tensor cores (no counterpart in the reference, which has no learned
 * part): gw[co][ci][t] = sum_v G[v][co] X[v + off(t)][ci] (t = 9 kz + 3 ky
 * + kx) and gb[co] = sum_v G[v][co], written (not accumulated) as FP32.
 * X: device bf16 [D][H][W][cin]; G: device bf16 [D][H][W][max(cout, 16)]
 * (the layer's output-gradient layout).  work: device scratch of at least
 * hp_conv3_wgrad_workspace() bytes, 16-byte aligned, for the per-CTA
 * partial sums, which a second kernel adds in a fixed order: the result is
 * the same bit for bit on every run.  W must be a multiple of 128 and
 * (cin, cout) among the compiled pairs.  *err (device int) receives nonzero
 * if a bounded device wait expired.
 */
int64_t hp_conv3_wgrad_workspace(int32_t D, int32_t H, int32_t W, int32_t cin, int32_t cout);
hp_status hp_conv3_wgrad(const void *X, const void *G, int32_t D, int32_t H, int32_t W,
                         int32_t cin, int32_t cout, float *gw, float *gb, void *work,
                         int64_t work_bytes, int32_t *err, void *stream);

/* ------------------------------------------------------------------ */
/* Learned torso preconditioner and flexible CG (no counterpart in the  */
/* reference, whose torso solver is Jacobi-PCG only)                    */
/* ------------------------------------------------------------------ */

/*
 * M(r) = omega D^-1 r + Q A_c^-1 Q^T r + P(s * CNN([R(D^-1 r) / s, geometry]))
 * with Q the aggregation over cubes of coarse_agg^3 voxels and A_c the
 * Galerkin coarse operator (dense inverse, at most HP_PC_MAX_COARSE
 * unknowns), and the network on a grid of half the torso resolution (see
 * csrc/precond.cu).  Torso dims must be multiples of (8, 8, 256).  label:
 * HOST unpadded material labels; sigma: HOST n_materials conductivities
 * (S/m, label 0 = air) and h_m the voxel size, as given to hp_torso_create;
 * pin_cell: padded flat index of the pinned voxel; init_params: HOST flat
 * parameter vector or NULL for a seeded random initialisation; coarse_agg:
 * 0 = automatic aggregate size, > 0 a fixed one, -1 = no coarse level.
 */
#define HP_PC_MAX_COARSE 2048
typedef struct {
  int32_t ni, nj, nk;
  const uint8_t *label;
  int32_t n_materials;
  int64_t pin_cell;
  float omega;
  uint64_t seed;
  const float *init_params;
  const double *sigma;
  double h_m;
  int32_t coarse_agg;
} HpPrecondDesc;

typedef struct HpPrecond HpPrecond;

hp_status hp_precond_create(const HpPrecondDesc *desc, HpPrecond **out, void *stream);
/* z = M(r) over the padded torso grid (device arrays: label uint8, invd and
 * r fp32, z fp32 out); use_net = 0 applies the Jacobi and coarse terms only. */
hp_status hp_precond_apply(HpPrecond *h, const uint8_t *label, const float *invd, const float *r,
                           float *z, int32_t use_net, void *stream);
/* One training step on the pair (r, e) (padded device fp32 arrays, A e = r):
 * forward, loss L = 1 - (r.z)^2 / ((z.A z)(r.e)) with z = M(r) (the error
 * energy one optimal step along z leaves), backward, and an Adam step of
 * size lr (lr = 0: gradients only).  *loss_out (host) receives the loss. */
hp_status hp_precond_train_step(HpPrecond *h, const uint8_t *label, const float *invd,
                                const float *r, const float *e, float lr, float *loss_out,
                                void *stream);
/* Flat FP32 parameters / last gradients to or from host memory (set = 1
 * uploads host_params); *n receives the parameter count. */
hp_status hp_precond_params(HpPrecond *h, float *host_params, float *host_grads, int64_t *n,
                            int32_t set, void *stream);
/* Network output of the last forward (half-resolution grid, fp32), the
 * input scale s and the device error flag, to host memory. */
hp_status hp_precond_output(HpPrecond *h, float *host_y, float *host_scale, int32_t *host_err,
                            void *stream);
/* Aggregate edge length and number of coarse unknowns (0, 0: no coarse level). */
hp_status hp_precond_coarse_info(const HpPrecond *h, int32_t *agg, int32_t *n_coarse);
hp_status hp_precond_destroy(HpPrecond *h);

/* Device pointers of a torso handle's padded arrays (for the preconditioner
 * and for tests). */
typedef struct {
  int32_t ni, nj, nk;
  int64_t n_cells, pin_cell;
  const uint8_t *label;
  const float *invd;
  float *r;
  double *x;
  float *b;
} HpTorsoArrays;
hp_status hp_torso_arrays(HpTorso *h, HpTorsoArrays *out);

/* Flexible CG with the learned preconditioner for one frame, judged by the
 * same FP64 true relative residual <= tol.  use_net = 0 runs the same
 * solver without the network (Jacobi + coarse level); use_net = k in
 * {1, 2, 4} adds the network term on every k-th iteration (flexible CG
 * admits a preconditioner that varies between iterations).  If a run with the
 * network has not converged after fallback_iter iterations, stagnates or
 * breaks down, FCG restarts from the current iterate without the network
 * (stats->restarts += 100; up to max(fallback_iter, 1000) iterations); if
 * that fails as well, plain Jacobi-PCG finishes the frame
 * (stats->restarts += 1000).  A small fallback_iter thus limits the network
 * to the first iterations of every frame. */
hp_status hp_torso_solve_frame_fcg(HpTorso *h, HpPrecond *p, const float *vm,
                                   int32_t vm_on_device, float *out, int32_t out_on_device,
                                   double tol, int32_t max_iter, int32_t fallback_iter,
                                   int32_t use_net, HpSolveStats *stats, void *stream);

/* Trains the preconditioner on residual/error pairs generated by the plain
 * solver: for each of n_frames frames (vm_frames: device fp32, frame f at
 * vm_frames + f * frame_stride) the frame is solved to tol_exact (warm
 * start from the previous frame), then for each k in ks (host, n_ks values)
 * plain PCG is restarted from the warm start for k iterations and the pair
 * (r_k, x* - x_k) gives `repeats` Adam steps of size lr.  loss_hist (host,
 * n_frames * n_ks * repeats) receives the losses. */
hp_status hp_torso_train_precond(HpTorso *h, HpPrecond *p, const float *vm_frames,
                                 int64_t frame_stride, int32_t n_frames, const int32_t *ks,
                                 int32_t n_ks, int32_t repeats, float lr, double tol_exact,
                                 float *loss_hist, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* HRDAYA_B200_H */
