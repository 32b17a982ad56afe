// Device kernels of the BiCGSTAB solve phase (sm_100a).
//
// One BiCGSTAB iteration of the reference (AFIIM/src/bicgstab.cpp:168-275) is nine
// launches here, each a single pass over HBM with the BLAS-1 work and the scalar
// recurrences fused in:
//   K1 tm = IDv o (H p)                 spmv, scale epilogue        (:172-173)
//   K2 pc = G tm,  sum pc^2             spmv, norm epilogue         (:175, :201)
//   K3 v = A pc,   alpha = m1/(r0.v)    spmv, dot epilogue          (:178, :181)
//   K4 s = r - alpha v, sum r^2, x^2    stream                      (:184-185, :201, :216)
//   K5 tm = IDv o (H s)                 spmv, scale epilogue        (:189-190)
//   K6 sc = G tm                        spmv                        (:192)
//   K7 t = A sc,   omega = t.s / t.t    spmv, 2-dot epilogue        (:195, :198)
//   K8 x += alpha pc + omega sc, r = s - omega t, m1 = r0.r, tests  (:207-267)
//   K9 p = r + beta (p - omega v)                                   (:270-271)
// Reductions are deterministic: each block reduces in a fixed tree, writes one partial,
// and the last block to finish (ticket counter) sums the partials in block order and
// applies the scalar step. A kernel launched after the solve finished returns at once
// (st->done), so iterations can be launched ahead of the host's convergence check.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

namespace fiim {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

// Device-resident scalars of one solve.
struct DState {
    double ro, rc, m1, m2, alpha, omega, beta, tol, eps;
    double pc2, x2, r2;        // ||pc||^2, ||x||^2, ||r||^2 of the current iteration
    double ts, tt, r0v;        // last dot products (inspection)
    int iter, nmax, stag, msteps, maxmsteps, info, done, alpha_guard;
    unsigned int ticket;       // last-block counter, reset by the last block
    int loops;                 // iteration bodies run by the device loop (guard + accounting)
};

template <typename V>
struct CsrView {
    const int *__restrict__ rp;
    const int *__restrict__ ci;
    const V *__restrict__ v;
    int n;
};

// ---------------------------------------------------------------- loads
// Matrix streams are read once per pass: evict-first so the vectors stay in L2.
__device__ __forceinline__ double ldm(const double *p) { return __ldcs(p); }
__device__ __forceinline__ float ldm(const float *p) { return __ldcs(p); }
__device__ __forceinline__ float ldm(const __nv_bfloat16 *p) {
    const unsigned short u = __ldcs(reinterpret_cast<const unsigned short *>(p));
    return __bfloat162float(__ushort_as_bfloat16(u));
}
__device__ __forceinline__ int ldi(const int *p) { return __ldcs(p); }
// Gathered vector entries: read-only path, cached.
template <typename X>
__device__ __forceinline__ X ldx(const X *p) { return __ldg(p); }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ---------------------------------------------------------------- reduction tail
// Reduce NR per-thread values over the grid. Every block must call it (uniformly).
// The last block calls op.finish(st, totals) from thread 0.
template <int NR, class Op>
__device__ __forceinline__ void grid_reduce(double (&v)[NR], double *__restrict__ partials,
                                            DState *st, const Op &op) {
    __shared__ double sm[kWarps][NR];
    __shared__ int last;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < NR; ++j) v[j] = warp_sum(v[j]);
    if (lane == 0)
#pragma unroll
        for (int j = 0; j < NR; ++j) sm[w][j] = v[j];
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int j = 0; j < NR; ++j) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < kWarps; ++k) s += sm[k][j];
            partials[(size_t)blockIdx.x * NR + j] = s;
        }
        __threadfence();
        const unsigned t = atomicAdd(&st->ticket, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double acc[NR];
#pragma unroll
    for (int j = 0; j < NR; ++j) acc[j] = 0.0;
    for (int k = threadIdx.x; k < (int)gridDim.x; k += kThreads)
#pragma unroll
        for (int j = 0; j < NR; ++j) acc[j] += __ldcg(partials + (size_t)k * NR + j);
#pragma unroll
    for (int j = 0; j < NR; ++j) acc[j] = warp_sum(acc[j]);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int j = 0; j < NR; ++j) sm[w][j] = acc[j];
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot[NR];
#pragma unroll
        for (int j = 0; j < NR; ++j) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < kWarps; ++k) s += sm[k][j];
            tot[j] = s;
        }
        st->ticket = 0u;
        op.finish(st, tot);
    }
}

// ---------------------------------------------------------------- SpMV epilogues
// emit(row, sum, red) stores the row result and adds its share to the reductions.
struct EpiStore {
    static constexpr int NR = 1;   // unused slot (arrays need a positive size)
    static constexpr bool REDUCES = false;
    static constexpr bool GATED = true;    // returns at once when the solve is done
    double *y;
    __device__ void emit(long i, double s, double (&)[NR]) const { y[i] = s; }
    __device__ void finish(DState *, const double *) const {}
};
struct EpiScale {                  // y = d o (M x): the D^{-1} scaling of the preconditioner
    static constexpr int NR = 1;
    static constexpr bool REDUCES = false;
    static constexpr bool GATED = true;    // returns at once when the solve is done
    double *y;
    const double *__restrict__ d;
    __device__ void emit(long i, double s, double (&)[NR]) const { y[i] = __ldg(d + i) * s; }
    __device__ void finish(DState *, const double *) const {}
};
struct EpiNorm {                   // y = M x, ||y||^2 -> st->pc2 (stagnation test)
    static constexpr int NR = 1;
    static constexpr bool REDUCES = true;
    static constexpr bool GATED = true;    // returns at once when the solve is done
    double *y;
    __device__ void emit(long i, double s, double (&r)[NR]) const { y[i] = s; r[0] += s * s; }
    __device__ void finish(DState *st, const double *t) const { st->pc2 = t[0]; }
};
struct EpiAlpha {                  // v = A pc, alpha = m1 / (r0 . v)
    static constexpr int NR = 1;
    static constexpr bool REDUCES = true;
    static constexpr bool GATED = true;    // returns at once when the solve is done
    double *y;
    const double *__restrict__ r0;
    __device__ void emit(long i, double s, double (&r)[NR]) const {
        y[i] = s;
        r[0] += __ldg(r0 + i) * s;
    }
    __device__ void finish(DState *st, const double *t) const {
        st->r0v = t[0];
        st->alpha = st->m1 / t[0];
        // ACIFIM/src/bicgstab.cpp:208-213: a non-finite alpha ends the solve with info 3.
        if (st->alpha_guard && !isfinite(st->alpha)) {
            st->iter = st->nmax;
            st->info = 3;
            st->done = 1;
        }
    }
};
struct EpiOmega {                  // t = A sc, omega = (t . s) / (t . t)
    static constexpr int NR = 2;
    static constexpr bool REDUCES = true;
    static constexpr bool GATED = true;    // returns at once when the solve is done
    double *y;
    const double *__restrict__ sv;
    __device__ void emit(long i, double s, double (&r)[NR]) const {
        y[i] = s;
        r[0] += s * __ldg(sv + i);
        r[1] += s * s;
    }
    __device__ void finish(DState *st, const double *t) const {
        st->ts = t[0];
        st->tt = t[1];
        st->omega = t[0] / t[1];
    }
};

struct FinInit;
// Fused start of the solve (AFIIM/src/bicgstab.cpp:151-161): with s = (A x)_i,
// p = b - s; r0 = p; r = p; sum r0^2 -> ro, m1 = ro^2, rc = ro.
struct EpiInit {
    static constexpr int NR = 1;
    static constexpr bool REDUCES = true;
    static constexpr bool GATED = true;    // returns at once when the solve is done
    const double *__restrict__ b;
    double *p, *r0, *r;
    __device__ void emit(long i, double s, double (&red)[NR]) const {
        const double pi = b[i] + (-1.0) * s;
        p[i] = pi;
        r0[i] = pi;
        r[i] = pi;
        red[0] += pi * pi;
    }
    __device__ void finish(DState *st, const double *t) const;
};
// True residual r = b - A x in FP64, sum r^2 and sum b^2 -> st->ts, st->tt.
struct EpiResid {
    static constexpr int NR = 2;
    static constexpr bool REDUCES = true;
    static constexpr bool GATED = false;  // runs after the solve has finished
    const double *__restrict__ b;
    double *r;
    __device__ void emit(long i, double s, double (&red)[NR]) const {
        const double bi = b[i], ri = bi - s;
        if (r) r[i] = ri;
        red[0] += ri * ri;
        red[1] += bi * bi;
    }
    __device__ void finish(DState *st, const double *t) const {
        st->ts = t[0];
        st->tt = t[1];
    }
};

// ACIFIM mode 'C' pieces (ACIFIM/src/bicgstab.cpp:395-420).
struct EpiSubFrom {                // y = a - (M x)            (vdSub after a product)
    static constexpr int NR = 1;
    static constexpr bool REDUCES = false;
    static constexpr bool GATED = true;    // returns at once when the solve is done
    double *y;
    const double *__restrict__ a;
    __device__ void emit(long i, double s, double (&)[NR]) const { y[i] = a[i] - s; }
    __device__ void finish(DState *, const double *) const {}
};
struct EpiAccum {                  // y = (M x) + y            (mkl_sparse_d_mv with beta = 1)
    static constexpr int NR = 1;
    static constexpr bool REDUCES = false;
    static constexpr bool GATED = true;    // returns at once when the solve is done
    double *y;
    __device__ void emit(long i, double s, double (&)[NR]) const { y[i] = s + y[i]; }
    __device__ void finish(DState *, const double *) const {}
};
struct EpiAccumScale {             // y = (M x) + y; z = y o d (last relaxation step, then vdMul)
    static constexpr int NR = 1;
    static constexpr bool REDUCES = false;
    static constexpr bool GATED = true;    // returns at once when the solve is done
    double *y, *z;
    const double *__restrict__ d;
    __device__ void emit(long i, double s, double (&)[NR]) const {
        const double t = s + y[i];
        y[i] = t;
        z[i] = t * __ldg(d + i);
    }
    __device__ void finish(DState *, const double *) const {}
};
struct EpiAccumNorm {              // y = (M x) + y, ||y||^2 -> st->pc2
    static constexpr int NR = 1;
    static constexpr bool REDUCES = true;
    static constexpr bool GATED = true;    // returns at once when the solve is done
    double *y;
    __device__ void emit(long i, double s, double (&r)[NR]) const {
        const double t = s + y[i];
        y[i] = t;
        r[0] += t * t;
    }
    __device__ void finish(DState *st, const double *t) const { st->pc2 = t[0]; }
};

// ---------------------------------------------------------------- CSR SpMV
// VEC lanes per row (2..32), 32/VEC rows per warp, grid-stride over row groups so a
// fixed grid (a multiple of the SM count) covers any n. Column indices and values
// are loaded coalesced across the lanes; x is gathered through the read-only path.
// FILL 0 uses every stored entry; 1 keeps col >= row and 2 keeps col <= row (MKL's
// TRIANGULAR descriptors) for callers whose factors were not filtered at upload.
template <int VEC, typename V, typename Epi, int FILL = 0>
static __global__ void __launch_bounds__(kThreads)
k_spmv(CsrView<V> M, const double *__restrict__ x, Epi epi, DState *st,
       double *__restrict__ partials) {
    if (Epi::GATED && st != nullptr && st->done) return;
    constexpr int RPW = 32 / VEC;
    const int lane = threadIdx.x & 31;
    const int sub = lane / VEC, lir = lane % VEC;
    const long warp = ((long)blockIdx.x * kThreads + threadIdx.x) >> 5;
    const long nwarps = ((long)gridDim.x * kThreads) >> 5;
    double red[Epi::NR];
#pragma unroll
    for (int j = 0; j < Epi::NR; ++j) red[j] = 0.0;
    for (long base = warp * RPW; base < M.n; base += nwarps * RPW) {
        const long row = base + sub;
        double s = 0.0;
        if (row < M.n) {
            const int beg = __ldg(M.rp + row), end = __ldg(M.rp + row + 1);
            for (int k = beg + lir; k < end; k += VEC) {
                const int c = ldi(M.ci + k);
                const double a = (double)ldm(M.v + k);
                if (FILL == 1 && c < row) continue;
                if (FILL == 2 && c > row) continue;
                s = fma(a, ldx(x + c), s);
            }
        }
#pragma unroll
        for (int o = VEC / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (row < M.n && lir == 0) epi.emit(row, s, red);
    }
    if constexpr (Epi::REDUCES) grid_reduce<Epi::NR>(red, partials, st, epi);
}

// ---------------------------------------------------------------- streaming kernels
// Grid-stride loop shared by the elementwise kernels.
#define FIIM_FOR_ROWS(i, n) \
    for (long i = (long)blockIdx.x * kThreads + threadIdx.x; i < (n); i += (long)gridDim.x * kThreads)

struct FinInit {   // ro = ||r0||, m1 = ro^2, rc = ro (AFIIM/src/bicgstab.cpp:161-165)
    __device__ void finish(DState *st, const double *t) const {
        st->ro = sqrt(t[0]);
        st->m1 = st->ro * st->ro;
        st->rc = st->ro;
        st->iter = 0;
        st->stag = 0;
        st->msteps = 0;
        if (st->nmax <= 0) {
            st->done = 1;
            if (st->nmax == 0) st->info = 3;
        }
    }
};

__device__ inline void EpiInit::finish(DState *st, const double *t) const { FinInit{}.finish(st, t); }

struct FinS {
    __device__ void finish(DState *st, const double *t) const {
        st->r2 = t[0];
        st->x2 = t[1];
    }
};

// s = r - alpha v; ||r||^2 (the residual norm the reference tests, before r is
// updated: AFIIM/src/bicgstab.cpp:216) and ||x||^2 (stagnation test, :201).
static __global__ void __launch_bounds__(kThreads)
k_update_s(long n, const double *__restrict__ r, const double *__restrict__ v,
           const double *__restrict__ x, double *__restrict__ s, DState *st,
           double *__restrict__ partials) {
    if (st->done) return;
    const double na = -st->alpha;
    double red[2] = {0.0, 0.0};
    FIIM_FOR_ROWS(i, n) {
        const double ri = r[i], xi = x[i];
        s[i] = ri + na * v[i];
        red[0] += ri * ri;
        red[1] += xi * xi;
    }
    grid_reduce<2>(red, partials, st, FinS{});
}

// Termination tests and the beta recurrence (AFIIM/src/bicgstab.cpp:201-274).
struct FinControl {
    __device__ void finish(DState *st, const double *t) const {
        const double a = st->alpha, om = st->omega;
        if (fabs(a) * sqrt(st->pc2) < st->eps * sqrt(st->x2)) st->stag++;   // :201-204
        else st->stag = 0;
        const double prc = st->rc;                                           // :213
        st->rc = sqrt(st->r2);                                               // :216
        if (prc < st->rc) st->msteps++;                                      // :219-222
        else st->msteps = 0;
        if (st->msteps >= st->maxmsteps) { st->info = 1; st->done = 1; return; }  // :225
        if (st->stag >= 3) { st->info = 2; st->done = 1; return; }                // :237
        if (st->rc < st->tol * st->ro) { st->info = 0; st->done = 1; return; }    // :249
        st->m2 = st->m1;                                                     // :262
        st->m1 = t[0];                                                       // :264
        st->beta = st->m1 * a / (om * st->m2);                               // :267
        st->iter++;                                                          // :274
        if (st->iter >= st->nmax) { st->info = 3; st->done = 1; }            // :168,277
    }
};

// x += alpha pc; x += omega sc; r = s - omega t; sum r0 . r; then the tests.
static __global__ void __launch_bounds__(kThreads)
k_update_xr(long n, const double *__restrict__ pc, const double *__restrict__ sc,
            const double *__restrict__ s, const double *__restrict__ t,
            const double *__restrict__ r0, double *__restrict__ x, double *__restrict__ r,
            DState *st, double *__restrict__ partials) {
    if (st->done) return;
    const double a = st->alpha, om = st->omega;
    double red[1] = {0.0};
    FIIM_FOR_ROWS(i, n) {
        double xi = x[i];
        xi = xi + a * pc[i];
        xi = xi + om * sc[i];
        x[i] = xi;
        const double ri = s[i] + (-om) * t[i];
        r[i] = ri;
        red[0] += r0[i] * ri;
    }
    grid_reduce<1>(red, partials, st, FinControl{});
}

// p = (-beta omega) v + beta p; p += r (AFIIM/src/bicgstab.cpp:270-271).
// In the device-driven loop this is the last kernel of the body: block 0 counts the
// body, trips a guard (info -5) should the body ever run past nmax + 2 times, and
// sets the WHILE node's condition to continue only while the solve is not done.
static __global__ void __launch_bounds__(kThreads)
k_update_p(long n, const double *__restrict__ r, const double *__restrict__ v,
           double *__restrict__ p, DState *st, cudaGraphConditionalHandle h, int cond) {
    if (cond && blockIdx.x == 0 && threadIdx.x == 0) {
        const int loops = ++st->loops;
        if (!st->done && loops > st->nmax + 2) {
            st->info = -5;
            st->done = 1;
        }
        cudaGraphSetConditional(h, st->done ? 0u : 1u);
    }
    if (st->done) return;
    const double b = st->beta, c = -st->beta * st->omega;
    FIIM_FOR_ROWS(i, n) { p[i] = (c * v[i] + b * p[i]) + r[i]; }
}

// Count entries of a CSR matrix outside the kept triangle (upper: col < row is outside;
// lower: col > row is outside).
static __global__ void k_count_outside(int n, const int *__restrict__ rp, const int *__restrict__ ci,
                                int upper, unsigned long long *count) {
    unsigned long long c = 0;
    FIIM_FOR_ROWS(i, n) {
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            const int j = ci[k];
            c += upper ? (j < i) : (j > i);
        }
    }
    if (c) atomicAdd(count, c);
}

}  // namespace fiim
