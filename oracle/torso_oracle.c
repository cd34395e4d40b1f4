/*
 * ORACLE -- test infrastructure, not product code.
 *
 * FP64 Jacobi-preconditioned CG over an assembled CSR matrix, threaded with
 * pthreads: the reference's per-frame torso solve (_pcg_gpu,
 * ecg/functions/compute_bspm.py:164-263: x0 = warm start, r = b - A x0,
 * z = M^-1 r, p = z; alpha = rz / pAp, x += alpha p, r -= alpha Ap,
 * z = M^-1 r, beta = rz_new / rz, p = z + beta p) run entirely in FP64 with
 * the relative-residual stop ||r|| <= tol ||b||.  The recursive residual only
 * proposes convergence: the true residual b - A x is then evaluated and, if
 * it misses the tolerance, becomes the new r and CG restarts.  Used by
 * tests/ and bench.py's CPU legs to judge the GPU's torso potentials and to
 * time the reference method on the host cores.  Reductions are summed per
 * thread over fixed row ranges and then in thread order (deterministic for a
 * given thread count).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

int orc_num_threads(void);

typedef struct {
    int64_t n;
    const int64_t *ptr; const int32_t *idx; const double *val;
    const double *b, *minv;
    double *x, *r, *z, *p, *ap;
    int nw;                      /* worker threads; the caller coordinates */
    pthread_barrier_t bar;       /* nw workers + the caller */
    double part[256][3];
    double alpha, beta;          /* written by the caller between phases */
    int phase;
} pcg_ctx;
typedef struct { pcg_ctx *c; int w; } pcg_arg;

enum { PH_TRUE_RES = 1, PH_AP = 2, PH_UPDATE = 3, PH_DIR = 4, PH_EXIT = 5 };

/* worker w owns rows [n w / nw, n (w + 1) / nw) */
static void *pcg_worker(void *pa) {
    pcg_arg *a = (pcg_arg *)pa;
    pcg_ctx *c = a->c;
    const int64_t lo = c->n * a->w / c->nw, hi = c->n * (a->w + 1) / c->nw;
    for (;;) {
        pthread_barrier_wait(&c->bar);
        const int ph = c->phase;
        if (ph == PH_EXIT) break;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
        if (ph == PH_TRUE_RES) {
            /* r = b - A x, z = M^-1 r, p = z; sums ||r||^2, r.z, ||b||^2 */
            for (int64_t i = lo; i < hi; ++i) {
                double ax = 0.0;
                for (int64_t q = c->ptr[i]; q < c->ptr[i + 1]; ++q) ax += c->val[q] * c->x[c->idx[q]];
                const double ri = c->b[i] - ax, zi = c->minv[i] * ri;
                c->r[i] = ri; c->z[i] = zi; c->p[i] = zi;
                s0 += ri * ri; s1 += ri * zi; s2 += c->b[i] * c->b[i];
            }
        } else if (ph == PH_AP) {
            for (int64_t i = lo; i < hi; ++i) {
                double ap = 0.0;
                for (int64_t q = c->ptr[i]; q < c->ptr[i + 1]; ++q) ap += c->val[q] * c->p[c->idx[q]];
                c->ap[i] = ap;
                s0 += c->p[i] * ap;
            }
        } else if (ph == PH_UPDATE) {
            const double al = c->alpha;
            for (int64_t i = lo; i < hi; ++i) {
                c->x[i] += al * c->p[i];
                const double ri = c->r[i] - al * c->ap[i], zi = c->minv[i] * ri;
                c->r[i] = ri; c->z[i] = zi;
                s0 += ri * ri; s1 += ri * zi;
            }
        } else if (ph == PH_DIR) {
            const double be = c->beta;
            for (int64_t i = lo; i < hi; ++i) c->p[i] = c->z[i] + be * c->p[i];
        }
        c->part[a->w][0] = s0; c->part[a->w][1] = s1; c->part[a->w][2] = s2;
        pthread_barrier_wait(&c->bar);
    }
    return NULL;
}

/* the caller releases the workers into phase ph and sums their partials in
 * worker order */
static void run_phase(pcg_ctx *c, int ph, double *sums) {
    c->phase = ph;
    pthread_barrier_wait(&c->bar);
    pthread_barrier_wait(&c->bar);
    sums[0] = sums[1] = sums[2] = 0.0;
    for (int w = 0; w < c->nw; ++w) {
        sums[0] += c->part[w][0]; sums[1] += c->part[w][1]; sums[2] += c->part[w][2];
    }
}

/*
 * Solves A x = b (n rows, CSR with int64 row pointers, int32 columns) from
 * the start x (in place) to ||b - A x|| <= tol ||b|| (true residual), at
 * most max_iter CG iterations in all.  minv = 1 / diag(A).  out[0] =
 * iterations, out[1] = true relative residual, out[2] = restarts.  Returns
 * 0, or -2 when memory ran out.
 */
int orc_csr_pcg(int64_t n, const int64_t *ptr, const int32_t *idx, const double *val,
                const double *minv, const double *b, double *x, double tol,
                int64_t max_iter, double *out) {
    pcg_ctx *c = (pcg_ctx *)calloc(1, sizeof(pcg_ctx));
    if (!c) return -2;
    c->n = n; c->ptr = ptr; c->idx = idx; c->val = val; c->b = b; c->minv = minv; c->x = x;
    c->r = (double *)malloc(sizeof(double) * n);
    c->z = (double *)malloc(sizeof(double) * n);
    c->p = (double *)malloc(sizeof(double) * n);
    c->ap = (double *)malloc(sizeof(double) * n);
    if (!c->r || !c->z || !c->p || !c->ap) {
        free(c->r); free(c->z); free(c->p); free(c->ap); free(c);
        return -2;
    }
    int nw = orc_num_threads();
    if (nw > 256) nw = 256;
    if (n < 65536) nw = 1;
    c->nw = nw;
    pthread_barrier_init(&c->bar, NULL, nw + 1);
    pthread_t th[256];
    pcg_arg args[256];
    for (int w = 0; w < nw; ++w) {
        args[w].c = c; args[w].w = w;
        pthread_create(&th[w], NULL, pcg_worker, &args[w]);
    }
    double s[3];
    int64_t it = 0, restarts = 0;
    double rel = INFINITY;
    for (;;) {
        run_phase(c, PH_TRUE_RES, s);
        const double bnorm = sqrt(s[2]);
        if (bnorm == 0.0) { rel = 0.0; break; }
        rel = sqrt(s[0]) / bnorm;
        if (rel <= tol || it >= max_iter || restarts >= 20) break;
        if (it > 0) ++restarts;
        double rz = s[1];
        while (it < max_iter) {
            run_phase(c, PH_AP, s);
            const double pap = s[0];
            if (fabs(pap) < 1e-300) break;
            c->alpha = rz / pap;
            run_phase(c, PH_UPDATE, s);
            ++it;
            if (sqrt(s[0]) <= tol * bnorm) break;
            c->beta = s[1] / rz;
            rz = s[1];
            run_phase(c, PH_DIR, s);
        }
    }
    c->phase = PH_EXIT;
    pthread_barrier_wait(&c->bar);
    for (int w = 0; w < nw; ++w) pthread_join(th[w], NULL);
    pthread_barrier_destroy(&c->bar);
    out[0] = (double)it; out[1] = rel; out[2] = (double)restarts;
    free(c->r); free(c->z); free(c->p); free(c->ap); free(c);
    return 0;
}
