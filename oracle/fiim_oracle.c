/* ORACLE TEST INFRASTRUCTURE — not product code.
 *
 * Plain-C restatement of the reference's preconditioned BiCGSTAB solve phase.
 * Arithmetic is sequential, left to right, with no FMA contraction (built with
 * -ffp-contract=off), matching oracle/mkl_shim run on one thread, so that the
 * reference compiled against the shim and this file agree bit for bit.
 * Citations are paths inside the reference repository.
 */
#include "fiim_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static int keep(int fill, int i, int j) {
    if (fill == ORC_UPPER) return j >= i;
    if (fill == ORC_LOWER) return j <= i;
    return 1;
}

/* y = A x over the entries the fill mode keeps; each row summed in storage order.
 * Restates mkl_sparse_d_mv(NON_TRANSPOSE, 1.0, A, descr, x, 0.0, y) as called at
 * AFIIM/src/bicgstab.cpp:151,172,175,178 (GENERAL / TRIANGULAR LOWER / UPPER). */
void orc_csr_mv(int n, const int *Ai, const int *Aj, const double *Av, int fill,
                const double *x, double *y) {
    for (int i = 0; i < n; ++i) {
        double s = 0.0;
        for (int k = Ai[i]; k < Ai[i + 1]; ++k)
            if (keep(fill, i, Aj[k])) s += Av[k] * x[Aj[k]];
        y[i] = s;
    }
}

/* y = T^T x for the kept triangle T. Restates mkl_sparse_d_mv(TRANSPOSE, ..., G,
 * TRIANGULAR UPPER) at PDFIIM/src/bicgstab.cpp:190,207. */
void orc_csr_mv_trans(int n, const int *Ai, const int *Aj, const double *Av, int fill,
                      const double *x, double *y) {
    double *acc = (double *)calloc((size_t)n, sizeof(double));
    for (int i = 0; i < n; ++i)
        for (int k = Ai[i]; k < Ai[i + 1]; ++k)
            if (keep(fill, i, Aj[k])) acc[Aj[k]] += Av[k] * x[i];
    memcpy(y, acc, sizeof(double) * (size_t)n);
    free(acc);
}

/* y = A x where A is symmetric and only its upper triangle is stored. Restates the
 * SYMMETRIC + UPPER descriptor of PDFIIM/src/bicgstab.cpp:149-153. */
void orc_csr_mv_sym_upper(int n, const int *Ai, const int *Aj, const double *Av,
                          const double *x, double *y) {
    double *acc = (double *)calloc((size_t)n, sizeof(double));
    for (int i = 0; i < n; ++i)
        for (int k = Ai[i]; k < Ai[i + 1]; ++k) {
            const int j = Aj[k];
            if (j < i) continue;
            acc[i] += Av[k] * x[j];
            if (j != i) acc[j] += Av[k] * x[i];
        }
    memcpy(y, acc, sizeof(double) * (size_t)n);
    free(acc);
}

/* out = G * (IDv o (H * in)). AFIIM/src/bicgstab.cpp:172-175; ACIFIM/src/bicgstab.cpp:393-394,
 * 408-410 (apply, mode 'E'); PDFIIM/src/bicgstab.cpp:192-194. H is applied as TRIANGULAR
 * LOWER and G as TRIANGULAR UPPER (AFIIM/src/bicgstab.cpp:140-147). tm holds H*in scaled. */
void orc_prec_apply(int n, const int *Gi, const int *Gj, const double *Gv, const double *IDv,
                    const int *Hi, const int *Hj, const double *Hv, const double *in,
                    double *out, double *tm) {
    double *hp = (double *)malloc(sizeof(double) * (size_t)n);
    orc_csr_mv(n, Hi, Hj, Hv, ORC_LOWER, in, hp);
    for (int i = 0; i < n; ++i) tm[i] = IDv[i] * hp[i];       /* vdMul(n, IDv, pc, tm) */
    orc_csr_mv(n, Gi, Gj, Gv, ORC_UPPER, tm, out);
    free(hp);
}

/* Symmetric PDFIIM form out = G * (IDv o (G^T * in)), PDFIIM/src/bicgstab.cpp:189-194. */
void orc_prec_apply_sym(int n, const int *Gi, const int *Gj, const double *Gv,
                        const double *IDv, const double *in, double *out, double *tm) {
    double *hp = (double *)malloc(sizeof(double) * (size_t)n);
    orc_csr_mv_trans(n, Gi, Gj, Gv, ORC_UPPER, in, hp);
    for (int i = 0; i < n; ++i) tm[i] = IDv[i] * hp[i];
    orc_csr_mv(n, Gi, Gj, Gv, ORC_UPPER, tm, out);
    free(hp);
}

/* ACIFIM apply(), mode 'C' (ACIFIM/src/bicgstab.cpp:395-404,408,411-420): Richardson-coupled
 *   t1 = H b;  repeat nr-1: t1 += H (b - L t1)
 *   t2 = t1 o IDv
 *   x = G t2;  repeat nr-1: x += G (t2 - U x)
 * The '+=' forms are mkl_sparse_d_mv with beta = 1: y = 1*s + 1*y. */
void orc_prec_apply_combined(int n, int nr, const int *Gi, const int *Gj, const double *Gv,
                             const double *IDv, const int *Hi, const int *Hj, const double *Hv,
                             const int *Li, const int *Lj, const double *Lv, const int *Ui,
                             const int *Uj, const double *Uv, const double *in, double *out,
                             double *work) {
    double *t1 = work, *t2 = work + n, *t3 = work + 2 * (size_t)n;
    double *tmp = (double *)malloc(sizeof(double) * (size_t)n);
    orc_csr_mv(n, Hi, Hj, Hv, ORC_LOWER, in, t1);
    for (int it = 1; it < nr; ++it) {
        orc_csr_mv(n, Li, Lj, Lv, ORC_LOWER, t1, t2);
        for (int i = 0; i < n; ++i) t3[i] = in[i] - t2[i];  /* vdSub(n, b, t2, t3) */
        orc_csr_mv(n, Hi, Hj, Hv, ORC_LOWER, t3, tmp);
        for (int i = 0; i < n; ++i) t1[i] = tmp[i] + t1[i];
    }
    for (int i = 0; i < n; ++i) t2[i] = t1[i] * IDv[i];      /* vdMul(n, t1, IDv, t2) */
    orc_csr_mv(n, Gi, Gj, Gv, ORC_UPPER, t2, out);
    for (int it = 1; it < nr; ++it) {
        orc_csr_mv(n, Ui, Uj, Uv, ORC_UPPER, out, t1);
        for (int i = 0; i < n; ++i) t3[i] = t2[i] - t1[i];  /* vdSub(n, t2, t1, t3) */
        orc_csr_mv(n, Gi, Gj, Gv, ORC_UPPER, t3, tmp);
        for (int i = 0; i < n; ++i) out[i] = tmp[i] + out[i];
    }
    free(tmp);
}

/* Number of contiguous blocks the dot products and norms are split into. 1 (default) is
 * the left-to-right sum of a one-thread MKL shim; B > 1 reproduces the shim's OpenMP
 * reduction on B threads (oracle/mkl_shim/mkl_shim.cpp blocked_sum): B static blocks,
 * each summed left to right, then the partials added in block order. Used to sample
 * how the reference's iteration counts move with the summation order alone. */
static int g_dot_blocks = 1;

void orc_set_dot_blocks(int blocks) { g_dot_blocks = blocks > 1 ? blocks : 1; }

static double dot(int n, const double *x, const double *y) {
    if (g_dot_blocks <= 1) {
        double s = 0.0;
        for (int i = 0; i < n; ++i) s += x[i] * y[i];
        return s;
    }
    const long T = g_dot_blocks, q = n / T, r = n % T;
    double s = 0.0;
    for (long t = 0; t < T; ++t) {
        const long lo = t * q + (t < r ? t : r), hi = lo + q + (t < r ? 1 : 0);
        double part = 0.0;
        for (long i = lo; i < hi; ++i) part += x[i] * y[i];
        s += part;
    }
    return s;
}

static double nrm2(int n, const double *x) { return sqrt(dot(n, x, x)); }

/* The BiCGSTAB loop shared by the three packages:
 *   AFIIM  EPBiCGSTAB  AFIIM/src/bicgstab.cpp:87-297
 *   PDFIIM EPBiCGSTAB  PDFIIM/src/bicgstab.cpp:80-310 (issym: :145-153,189-192,206-209)
 *   ACIFIM PBiCGSTAB   ACIFIM/src/bicgstab.cpp:97-327 (non-finite alpha guard :208-213,
 *                      divergence window :132, apply() :372-428)
 * Step numbers below refer to AFIIM/src/bicgstab.cpp. */
int orc_bicgstab(int variant, int issym, char mode, int nr, int n, const int *Ai, const int *Aj,
                 const double *Av, const double *b, double tol, int NMAX, const int *Gi,
                 const int *Gj, const double *Gv, const double *IDv, const int *Hi,
                 const int *Hj, const double *Hv, const int *Li, const int *Lj,
                 const double *Lv, const int *Ui, const int *Uj, const double *Uv, double *x,
                 double *resval, int *iter, int *info) {
    if (variant == ORC_ACIFIM && mode != 'E' && mode != 'C') return -1;
    if (issym && variant != ORC_PDFIIM) return -1;
    const double eps = 1.11022302462516e-16;                         /* :108 */
    const int maxstagsteps = 3;                                      /* :112 */
    int stag = 0, msteps = 0, maxmsteps;
    if (variant == ORC_ACIFIM) {                                     /* ACIFIM :132 */
        int m = (n > 2000 ? n : 2000) / 50;
        maxmsteps = m < 40 ? m : 40;
    } else {                                                         /* :114 */
        int m = (n > 500 ? n : 500) / 50;
        maxmsteps = m < 20 ? m : 20;
    }
    const size_t sz = sizeof(double) * (size_t)n;
    double *p = malloc(sz), *r0 = malloc(sz), *r = malloc(sz), *v = malloc(sz), *s = malloc(sz);
    double *t = malloc(sz), *pc = malloc(sz), *sc = malloc(sz), *tm = malloc(sz);
    double *work = malloc(3 * sz + 1);
    double ro, a, om, m1, m2, rc, prc, beta;

    *iter = 0;
#define AMUL(xin, yout)                                                        \
    do {                                                                       \
        if (issym) orc_csr_mv_sym_upper(n, Ai, Aj, Av, xin, yout);             \
        else orc_csr_mv(n, Ai, Aj, Av, ORC_GENERAL, xin, yout);                \
    } while (0)
#define PREC(xin, yout)                                                        \
    do {                                                                       \
        if (issym) orc_prec_apply_sym(n, Gi, Gj, Gv, IDv, xin, yout, tm);      \
        else if (variant == ORC_ACIFIM && mode == 'C')                         \
            orc_prec_apply_combined(n, nr, Gi, Gj, Gv, IDv, Hi, Hj, Hv, Li, Lj, \
                                    Lv, Ui, Uj, Uv, xin, yout, work);          \
        else orc_prec_apply(n, Gi, Gj, Gv, IDv, Hi, Hj, Hv, xin, yout, tm);    \
    } while (0)

    AMUL(x, r);                                                      /* :151 r = A x */
    for (int i = 0; i < n; ++i) p[i] = b[i];                         /* :153 */
    for (int i = 0; i < n; ++i) p[i] += -1.0 * r[i];                 /* :154 p = b - r */
    memcpy(r0, p, sz);                                               /* :157 */
    memcpy(r, p, sz);                                                /* :158 */
    ro = nrm2(n, r0);                                                /* :161 */
    m1 = ro * ro;                                                    /* :162 */
    rc = ro;                                                         /* :165 */

    while (*iter < NMAX) {                                           /* :168 */
        PREC(p, pc);                                                 /* :172-175 */
        AMUL(pc, v);                                                 /* :178 */
        a = m1 / dot(n, r0, v);                                      /* :181 */
        if (variant == ORC_ACIFIM && !isfinite(a)) {                 /* ACIFIM :208-213 */
            *iter = NMAX;
            *info = 3;
            break;
        }
        memcpy(s, r, sz);                                            /* :184 */
        for (int i = 0; i < n; ++i) s[i] += -a * v[i];               /* :185 */
        PREC(s, sc);                                                 /* :189-192 */
        AMUL(sc, t);                                                 /* :195 */
        om = dot(n, t, s) / dot(n, t, t);                            /* :198 */
        if (fabs(a) * nrm2(n, pc) < eps * nrm2(n, x)) stag++;        /* :201-204 */
        else stag = 0;
        for (int i = 0; i < n; ++i) x[i] += a * pc[i];               /* :207 */
        for (int i = 0; i < n; ++i) x[i] += om * sc[i];              /* :210 */
        prc = rc;                                                    /* :213 */
        rc = nrm2(n, r);                                             /* :216 (old r) */
        if (prc < rc) msteps++;                                      /* :219-222 */
        else msteps = 0;
        if (msteps >= maxmsteps) { *info = 1; break; }               /* :225-234 */
        if (stag >= maxstagsteps) { *info = 2; break; }              /* :237-246 */
        if (rc < tol * ro) { *info = 0; break; }                     /* :249-255 */
        memcpy(r, s, sz);                                            /* :258 */
        for (int i = 0; i < n; ++i) r[i] += -om * t[i];              /* :259 */
        m2 = m1;                                                     /* :262 */
        m1 = dot(n, r0, r);                                          /* :264 */
        beta = m1 * a / (om * m2);                                   /* :267 */
        for (int i = 0; i < n; ++i) p[i] = -beta * om * v[i] + beta * p[i]; /* :270 */
        for (int i = 0; i < n; ++i) p[i] += 1.0 * r[i];              /* :271 */
        (*iter)++;                                                   /* :274 */
    }
    if (*iter == NMAX) *info = 3;                                    /* :277-282 */
    *resval = rc / ro;                                               /* :285 */
#undef AMUL
#undef PREC
    free(p); free(r0); free(r); free(v); free(s); free(t); free(pc); free(sc); free(tm);
    free(work);
    return 0;
}
