// Device kernels of the FP64 BiCGSTAB solve phase (sm_100a).
//
// One BiCGSTAB iteration of the reference (AFIIM/src/bicgstab.cpp:168-275) is nine
// launches, each one pass over HBM with the BLAS-1 work and the scalar recurrences
// fused in:
//   K1 tm = IDv o (H p)                 spmv, scale epilogue        (:172-173)
//   K2 pc = G tm,  sum pc^2             spmv, norm epilogue         (:175, :201)
//   K3 v = A pc,   alpha = m1/(r0.v)    spmv, dot epilogue          (:178, :181)
//   K4 s = r - alpha v, sum r^2, x^2    stream                      (:184-185, :201, :216)
//   K5 tm = IDv o (H s)                 spmv, scale epilogue        (:189-190)
//   K6 sc = G tm                        spmv                        (:192)
//   K7 t = A sc,   omega = t.s / t.t    spmv, 2-dot epilogue        (:195, :198)
//   K8 x += alpha pc + omega sc, r = s - omega t, m1 = r0.r, tests  (:207-267)
//   K9 p = r + beta (p - omega v)                                   (:270-271)
//
// Rounding: every vector the reference computes is computed here with the same
// operations in the same order: each SpMV row is summed left to right in storage
// order with the product rounded before the add (as the MKL restatement in the oracle
// and as a CSR loop without FMA contraction), and every axpy / axpby / vdMul rounds the
// products and sums separately (explicit __dmul_rn / __dadd_rn, never FMA). Given the
// same scalars, the GPU's vectors are bit-identical to the reference's. The scalars
// come from dot products and norms, whose summation order is parallel here (a fixed
// tree, deterministic run to run) and left to right in the reference; that is the only
// source of difference.
//
// Reductions: each block reduces in a fixed tree and writes one partial; the last
// block to finish (ticket counter) sums the partials in block order and applies the
// scalar step. A gated kernel launched after the solve finished returns at once
// (st->done), so iterations can run ahead of any host check.
#pragma once

#include <type_traits>
#include <utility>

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
    double ts, tt, r0v;        // last dot products (inspection; true residual after a solve)
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

// ---------------------------------------------------------------- launch dependencies
// Programmatic dependent launch: pdl_enter waits for the previous kernel in the stream to
// complete (its writes visible) before anything it produced is touched; pdl_release, once
// a CTA's main loop is done, lets the next kernel's CTAs be scheduled during this kernel's
// tail. Both are no-ops in a launch without the programmatic-serialization attribute.
__device__ __forceinline__ void pdl_enter() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// ---------------------------------------------------------------- loads
// Matrix streams are read once per pass: evict-first so the vectors stay in L2.
__device__ __forceinline__ double ldm(const double *p) { return __ldcs(p); }
__device__ __forceinline__ float ldm(const float *p) { return __ldcs(p); }
// A BF16 value is the upper half of the FP32 value it stands for: widening is a shift.
__device__ __forceinline__ float ldm(const __nv_bfloat16 *p) {
    const unsigned short u = __ldcs(reinterpret_cast<const unsigned short *>(p));
    return __uint_as_float((unsigned)u << 16);
}
__device__ __forceinline__ int ldi(const int *p) { return __ldcs(p); }
__device__ __forceinline__ int2 ldi2(const int *p) { return __ldcs(reinterpret_cast<const int2 *>(p)); }
__device__ __forceinline__ double2 ldm2(const double *p) { return __ldcs(reinterpret_cast<const double2 *>(p)); }
// Matrix values prefetched into registers stay in the form they were loaded in until they
// are used: an FP64 or FP32 pair as two values, a BF16 pair as one 32-bit word. Widening a
// BF16 value at load time would make the prefetching thread wait for the load there.
template <typename V>
struct ValPair;
template <>
struct ValPair<double> {
    using T = double2;
    __device__ static T load2(const double *p) { return __ldcs(reinterpret_cast<const double2 *>(p)); }
    __device__ static T load1(const double *p) { return make_double2(__ldcs(p), 0.0); }
    __device__ static T zero() { return make_double2(0.0, 0.0); }
    __device__ static double get(const T &t, int h) { return h ? t.y : t.x; }
};
template <>
struct ValPair<float> {
    using T = float2;
    __device__ static T load2(const float *p) { return __ldcs(reinterpret_cast<const float2 *>(p)); }
    __device__ static T load1(const float *p) { return make_float2(__ldcs(p), 0.f); }
    __device__ static T zero() { return make_float2(0.f, 0.f); }
    __device__ static float get(const T &t, int h) { return h ? t.y : t.x; }
};
template <>
struct ValPair<__nv_bfloat16> {   // the first value in the low half (little-endian)
    using T = unsigned;
    __device__ static T load2(const __nv_bfloat16 *p) { return __ldcs(reinterpret_cast<const unsigned *>(p)); }
    __device__ static T load1(const __nv_bfloat16 *p) {
        return (unsigned)__ldcs(reinterpret_cast<const unsigned short *>(p));
    }
    __device__ static T zero() { return 0u; }
    __device__ static float get(const T &t, int h) { return __uint_as_float(h ? (t & 0xffff0000u) : (t << 16)); }
};

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

// ---------------------------------------------------------------- scalar steps
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

// ---------------------------------------------------------------- SpMV epilogues
// emit(row, sum, red) stores the row result and adds its share to the reductions.
// GATED kernels return at once once the solve is done.
#define FIIM_EPI(nr, reduces, gated)              \
    static constexpr int NR = nr;                 \
    static constexpr bool REDUCES = reduces;      \
    static constexpr bool GATED = gated

template <typename E, typename = void>
struct HasPre : std::false_type {};
template <typename E>
struct HasPre<E, std::void_t<decltype(std::declval<const E &>().pre(0L))>> : std::true_type {};

struct EpiStore {                  // y = M x
    FIIM_EPI(1, false, true);
    double *y;
    __device__ void emit(long i, double s, double (&)[NR]) const { y[i] = s; }
    __device__ void finish(DState *, const double *) const {}
};
// Epilogues with a per-row operand also offer pre_ptr(), the operand array, pre(i), its
// load, and emit_pre(i, s, o, red); the CSR-stream SpMV forms load the operand together
// with the next row block's streams (HasPre).
struct EpiScale {                  // y = d o (M x): vdMul(n, IDv, pc, tm), AFIIM/src/bicgstab.cpp:173
    FIIM_EPI(1, false, true);
    double *y;
    const double *__restrict__ d;
    __device__ const double *pre_ptr() const { return d; }
    __device__ double pre(long i) const { return __ldg(d + i); }
    __device__ void emit_pre(long i, double s, double di, double (&)[NR]) const { y[i] = __dmul_rn(di, s); }
    __device__ void emit(long i, double s, double (&r)[NR]) const { emit_pre(i, s, pre(i), r); }
    __device__ void finish(DState *, const double *) const {}
};
struct EpiNorm {                   // y = M x, ||y||^2 -> st->pc2 (stagnation test)
    FIIM_EPI(1, true, true);
    double *y;
    __device__ void emit(long i, double s, double (&r)[NR]) const { y[i] = s; r[0] += s * s; }
    __device__ void finish(DState *st, const double *t) const { st->pc2 = t[0]; }
};
struct EpiAlpha {                  // v = A pc, alpha = m1 / (r0 . v)
    FIIM_EPI(1, true, true);
    double *y;
    const double *__restrict__ r0;
    __device__ const double *pre_ptr() const { return r0; }
    __device__ double pre(long i) const { return __ldg(r0 + i); }
    __device__ void emit_pre(long i, double s, double r0i, double (&r)[NR]) const {
        y[i] = s;
        r[0] += r0i * s;
    }
    __device__ void emit(long i, double s, double (&r)[NR]) const { emit_pre(i, s, pre(i), r); }
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
    FIIM_EPI(2, true, true);
    double *y;
    const double *__restrict__ sv;
    __device__ const double *pre_ptr() const { return sv; }
    __device__ double pre(long i) const { return __ldg(sv + i); }
    __device__ void emit_pre(long i, double s, double si, double (&r)[NR]) const {
        y[i] = s;
        r[0] += s * si;
        r[1] += s * s;
    }
    __device__ void emit(long i, double s, double (&r)[NR]) const { emit_pre(i, s, pre(i), r); }
    __device__ void finish(DState *st, const double *t) const {
        st->ts = t[0];
        st->tt = t[1];
        st->omega = t[0] / t[1];
    }
};
// Fused start of the solve (AFIIM/src/bicgstab.cpp:151-161): with s = (A x)_i,
// p = b + (-1) s; r0 = p; r = p; sum r0^2 -> ro, m1 = ro^2, rc = ro.
struct EpiInit {
    FIIM_EPI(1, true, true);
    const double *__restrict__ b;
    double *p, *r0, *r;
    __device__ void emit(long i, double s, double (&red)[NR]) const {
        const double pi = __dadd_rn(b[i], __dmul_rn(-1.0, s));
        p[i] = pi;
        r0[i] = pi;
        r[i] = pi;
        red[0] += pi * pi;
    }
    __device__ void finish(DState *st, const double *t) const { FinInit{}.finish(st, t); }
};
// True residual r = b - A x in FP64, sum r^2 and sum b^2 -> st->ts, st->tt. Runs after
// the solve has finished, so it is not gated.
struct EpiResid {
    FIIM_EPI(2, true, false);
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
    FIIM_EPI(1, false, true);
    double *y;
    const double *__restrict__ a;
    __device__ void emit(long i, double s, double (&)[NR]) const { y[i] = __dadd_rn(a[i], -s); }
    __device__ void finish(DState *, const double *) const {}
};
struct EpiAccum {                  // y = (M x) + y            (mkl_sparse_d_mv with beta = 1)
    FIIM_EPI(1, false, true);
    double *y;
    __device__ void emit(long i, double s, double (&)[NR]) const { y[i] = __dadd_rn(s, y[i]); }
    __device__ void finish(DState *, const double *) const {}
};
struct EpiAccumScale {             // y = (M x) + y; z = y o d (last relaxation step, then vdMul)
    FIIM_EPI(1, false, true);
    double *y, *z;
    const double *__restrict__ d;
    __device__ void emit(long i, double s, double (&)[NR]) const {
        const double t = __dadd_rn(s, y[i]);
        y[i] = t;
        z[i] = __dmul_rn(t, __ldg(d + i));
    }
    __device__ void finish(DState *, const double *) const {}
};
struct EpiAccumNorm {              // y = (M x) + y, ||y||^2 -> st->pc2
    FIIM_EPI(1, true, true);
    double *y;
    __device__ void emit(long i, double s, double (&r)[NR]) const {
        const double t = __dadd_rn(s, y[i]);
        y[i] = t;
        r[0] += t * t;
    }
    __device__ void finish(DState *st, const double *t) const { st->pc2 = t[0]; }
};

// ---------------------------------------------------------------- CSR-stream SpMV
// Rows are grouped at set-up into row blocks: consecutive rows, at most kThreads of
// them, whose entries total at most TILE - 1; a row of TILE or more entries is a block
// of its own. rb holds each block's first row and eb its first entry (nblk + 1 of each). A CTA
// takes row blocks in grid-stride order. For each block it streams the entries coalesced
// (columns and values with evict-first loads, x gathered through the read-only path),
// stores the rounded products v*x in shared memory, then each thread sums its own row's
// products left to right. A long row is summed by one thread over TILE-sized chunks,
// still in storage order.
//
// The loop is software-pipelined by one block: the next block's bounds, this thread's
// row offsets in it and its share of the column/value stream are loaded into registers
// before the barrier, so they are in flight while the current block's rows are summed.
// Narrow column stream (NARROW): 16-bit offsets from a per-row-block base column, built by
// k_narrow_cols when every block's columns span at most 65,536; 10 bytes per entry instead of
// 12. A thread keeps each prefetched pair of offsets as the 32-bit word it was loaded as and
// forms the columns only at the product, so no instruction waits on the prefetch.
struct NarrowCols {
    const short *__restrict__ d = nullptr;     // column - base of the entry's block
    const int *__restrict__ base = nullptr;    // per row block
};

template <bool NARROW, int PER>
struct ColRegs;
template <int PER>
struct ColRegs<false, PER> {
    int c[PER];
    __device__ void zero(int u) { c[2 * u] = c[2 * u + 1] = 0; }
    __device__ void load2(const int *ci, const NarrowCols &, int e, int u) {
        const int2 cc = ldi2(ci + e);
        c[2 * u] = cc.x;
        c[2 * u + 1] = cc.y;
    }
    __device__ void load1(const int *ci, const NarrowCols &, int e, int u) { c[2 * u] = ldi(ci + e); }
    __device__ int get(int u, int) const { return c[u]; }
};
template <int PER>
struct ColRegs<true, PER> {
    unsigned w[PER / 2];
    __device__ void zero(int u) { w[u] = 0u; }
    __device__ void load2(const int *, const NarrowCols &nc, int e, int u) {
        w[u] = __ldcs(reinterpret_cast<const unsigned *>(nc.d + e));
    }
    __device__ void load1(const int *, const NarrowCols &nc, int e, int u) {
        w[u] = (unsigned)__ldcs(reinterpret_cast<const unsigned short *>(nc.d + e));
    }
    __device__ int get(int u, int base) const {
        const unsigned v = w[u >> 1];
        return base + (int)(short)(unsigned short)((u & 1) ? (v >> 16) : (v & 0xffffu));
    }
};

template <int TILE, typename Epi, bool NARROW = false>
static __global__ void __launch_bounds__(kThreads)
k_spmv_rows(CsrView<double> M, const int *__restrict__ rb, const int *__restrict__ eb, int nblk,
            const double *__restrict__ x, Epi epi, DState *st, double *__restrict__ partials,
            NarrowCols nc = NarrowCols{}) {
    pdl_enter();
    if (Epi::GATED && st != nullptr && st->done) return;
    __shared__ double prod[TILE];
    constexpr int PER = TILE / kThreads;
    const int tid = (int)threadIdx.x;
    double red[Epi::NR];
#pragma unroll
    for (int j = 0; j < Epi::NR; ++j) red[j] = 0.0;
    int r0 = 0, r1 = 0, e0 = 0, e1 = 0, rbeg = 0, rend = 0, cbase = 0;
    double opnd = 0.0;   // the epilogue's operand for this thread's row (HasPre)
    // Entries are read in aligned pairs: thread tid holds entries a0 + 2 (tid + u kThreads)
    // + h of the window [a0, a0 + TILE), a0 = e0 rounded down to even. Row blocks have at
    // most TILE - 1 entries, so the window covers [e0, e1); a block that does not fit is a
    // single long row.
    ColRegs<NARROW, PER> c;
    double a[PER];
    auto fetch = [&](int blk) {
        r0 = __ldg(rb + blk);
        r1 = __ldg(rb + blk + 1);
        e0 = __ldg(eb + blk);
        e1 = __ldg(eb + blk + 1);
        if constexpr (NARROW) cbase = __ldg(nc.base + blk);
        rbeg = rend = 0;
        if (r0 + tid < r1) {
            rbeg = __ldg(M.rp + r0 + tid);
            rend = __ldg(M.rp + r0 + tid + 1);
            if constexpr (HasPre<Epi>::value) opnd = epi.pre(r0 + tid);
        }
        if (e1 - e0 < TILE) {
            const int a0 = e0 & ~1;
#pragma unroll
            for (int u = 0; u < PER / 2; ++u) {
                const int e = a0 + 2 * (tid + u * kThreads);
                c.zero(u);
                a[2 * u] = a[2 * u + 1] = 0.0;
                if (e + 1 < e1) {
                    c.load2(M.ci, nc, e, u);
                    const double2 aa = ldm2(M.v + e);
                    a[2 * u] = aa.x;
                    a[2 * u + 1] = aa.y;
                } else if (e < e1) {
                    c.load1(M.ci, nc, e, u);
                    a[2 * u] = ldm(M.v + e);
                }
            }
        }
    };
    if ((int)blockIdx.x < nblk) fetch(blockIdx.x);
    for (int blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
        const int nxt = blk + (int)gridDim.x;
        const int cr0 = r0, cr1 = r1, ce0 = e0, ce1 = e1, cb = rbeg - e0, ce = rend - e0, cbs = cbase;
        const double copnd = opnd;
        if (ce1 - ce0 < TILE) {
            const int a0 = ce0 & ~1;
#pragma unroll
            for (int u = 0; u < PER; ++u) {
                const int e = a0 + 2 * (tid + (u >> 1) * kThreads) + (u & 1);
                if (e >= ce0 && e < ce1) prod[e - ce0] = __dmul_rn(a[u], ldx(x + c.get(u, cbs)));
            }
            if (nxt < nblk) fetch(nxt);
            __syncthreads();
            if (cr0 + tid < cr1) {
                double s = 0.0;
                for (int k = cb; k < ce; ++k) s = __dadd_rn(s, prod[k]);
                if constexpr (HasPre<Epi>::value) epi.emit_pre(cr0 + tid, s, copnd, red);
                else epi.emit(cr0 + tid, s, red);
            }
            __syncthreads();
        } else {
            double s = 0.0;
            for (int c0 = ce0; c0 < ce1; c0 += TILE) {
                const int c1 = min(c0 + TILE, ce1);
                for (int e = c0 + tid; e < c1; e += kThreads) {
                    const int j = NARROW ? cbs + (int)__ldcs(nc.d + e) : ldi(M.ci + e);
                    prod[e - c0] = __dmul_rn(ldm(M.v + e), ldx(x + j));
                }
                __syncthreads();
                if (tid == 0)
                    for (int k = 0; k < c1 - c0; ++k) s = __dadd_rn(s, prod[k]);
                __syncthreads();
            }
            if (tid == 0) epi.emit(cr0, s, red);
            if (nxt < nblk) fetch(nxt);
        }
    }
    pdl_release();
    if constexpr (Epi::REDUCES) grid_reduce<Epi::NR>(red, partials, st, epi);
}

// Warp-block form of the CSR-stream SpMV: the same arithmetic as k_spmv_rows (rounded
// products staged in shared memory, each row summed left to right by one thread), with row
// blocks of at most 32 rows and WT - 1 entries that each warp takes on its own, in
// grid-stride order over the warps. A warp synchronises only with itself (__syncwarp), so
// the warps of a CTA do not wait for one another between blocks; the loop is pipelined by
// one block per warp, as in k_spmv_rows. A row of WT or more entries is a block of its own,
// summed by lane 0 over WT-sized chunks, still in storage order.
template <int WT, typename Epi, bool NARROW = false>
static __global__ void __launch_bounds__(kThreads)
k_spmv_warp(CsrView<double> M, const int *__restrict__ rb, const int *__restrict__ eb, int nblk,
            const double *__restrict__ x, Epi epi, DState *st, double *__restrict__ partials,
            NarrowCols nc = NarrowCols{}) {
    pdl_enter();
    if (Epi::GATED && st != nullptr && st->done) return;
    __shared__ double prod_all[kWarps][WT];
    constexpr int PER = WT / 32;
    const int lane = (int)threadIdx.x & 31, w = (int)threadIdx.x >> 5;
    double *prod = prod_all[w];
    const int gw = (int)blockIdx.x * kWarps + w, nw = (int)gridDim.x * kWarps;
    double red[Epi::NR];
#pragma unroll
    for (int j = 0; j < Epi::NR; ++j) red[j] = 0.0;
    int r0 = 0, r1 = 0, e0 = 0, e1 = 0, rbeg = 0, rend = 0, cbase = 0;
    double opnd = 0.0;
    ColRegs<NARROW, PER> c;
    double a[PER];
    auto fetch = [&](int blk) {
        r0 = __ldg(rb + blk);
        r1 = __ldg(rb + blk + 1);
        e0 = __ldg(eb + blk);
        e1 = __ldg(eb + blk + 1);
        if constexpr (NARROW) cbase = __ldg(nc.base + blk);
        rbeg = rend = 0;
        if (r0 + lane < r1) {
            rbeg = __ldg(M.rp + r0 + lane);
            rend = __ldg(M.rp + r0 + lane + 1);
            if constexpr (HasPre<Epi>::value) opnd = epi.pre(r0 + lane);
        }
        if (e1 - e0 < WT) {
            const int a0 = e0 & ~1;
#pragma unroll
            for (int u = 0; u < PER / 2; ++u) {
                const int e = a0 + 2 * (lane + u * 32);
                c.zero(u);
                a[2 * u] = a[2 * u + 1] = 0.0;
                if (e + 1 < e1) {
                    c.load2(M.ci, nc, e, u);
                    const double2 aa = ldm2(M.v + e);
                    a[2 * u] = aa.x;
                    a[2 * u + 1] = aa.y;
                } else if (e < e1) {
                    c.load1(M.ci, nc, e, u);
                    a[2 * u] = ldm(M.v + e);
                }
            }
        }
    };
    if (gw < nblk) fetch(gw);
    for (int blk = gw; blk < nblk; blk += nw) {
        const int nxt = blk + nw;
        const int cr0 = r0, cr1 = r1, ce0 = e0, ce1 = e1, cb = rbeg - e0, ce = rend - e0, cbs = cbase;
        const double copnd = opnd;
        if (ce1 - ce0 < WT) {
            const int a0 = ce0 & ~1;
#pragma unroll
            for (int u = 0; u < PER; ++u) {
                const int e = a0 + 2 * (lane + (u >> 1) * 32) + (u & 1);
                if (e >= ce0 && e < ce1) prod[e - ce0] = __dmul_rn(a[u], ldx(x + c.get(u, cbs)));
            }
            if (nxt < nblk) fetch(nxt);
            __syncwarp();
            if (cr0 + lane < cr1) {
                double s = 0.0;
                for (int k = cb; k < ce; ++k) s = __dadd_rn(s, prod[k]);
                if constexpr (HasPre<Epi>::value) epi.emit_pre(cr0 + lane, s, copnd, red);
                else epi.emit(cr0 + lane, s, red);
            }
            __syncwarp();
        } else {
            double s = 0.0;
            for (int c0 = ce0; c0 < ce1; c0 += WT) {
                const int c1 = min(c0 + WT, ce1);
                for (int e = c0 + lane; e < c1; e += 32) {
                    const int j = NARROW ? cbs + (int)__ldcs(nc.d + e) : ldi(M.ci + e);
                    prod[e - c0] = __dmul_rn(ldm(M.v + e), ldx(x + j));
                }
                __syncwarp();
                if (lane == 0)
                    for (int k = 0; k < c1 - c0; ++k) s = __dadd_rn(s, prod[k]);
                __syncwarp();
            }
            if (lane == 0) epi.emit(cr0, s, red);
            if (nxt < nblk) fetch(nxt);
        }
    }
    pdl_release();
    if constexpr (Epi::REDUCES) grid_reduce<Epi::NR>(red, partials, st, epi);
}

// Narrow column stream for k_spmv_rows: per row block, base = smallest column + 32768 and
// d[e] = column - base, when the block's columns span at most 65,536; otherwise *wide is set
// and the matrix keeps its 32-bit columns. One CTA per block, grid-stride.
static __global__ void __launch_bounds__(kThreads)
k_narrow_cols(const int *__restrict__ ci, const int *__restrict__ eb, int nblk, short *__restrict__ d,
              int *__restrict__ base, int *wide) {
    __shared__ int smin[kWarps], smax[kWarps];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
        const int e0 = eb[blk], e1 = eb[blk + 1];
        int lo = 0x7fffffff, hi = -0x7fffffff - 1;
        for (int e = e0 + (int)threadIdx.x; e < e1; e += kThreads) {
            lo = min(lo, ci[e]);
            hi = max(hi, ci[e]);
        }
        for (int o = 16; o > 0; o >>= 1) {
            lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        if (lane == 0) {
            smin[w] = lo;
            smax[w] = hi;
        }
        __syncthreads();
        lo = smin[0];
        hi = smax[0];
        for (int q = 1; q < kWarps; ++q) {
            lo = min(lo, smin[q]);
            hi = max(hi, smax[q]);
        }
        __syncthreads();
        if (e1 > e0 && (long)hi - (long)lo > 65535) {
            if (threadIdx.x == 0) atomicExch(wide, 1);
            continue;
        }
        const int b = e1 > e0 ? lo + 32768 : 0;
        if (threadIdx.x == 0) base[blk] = b;
        for (int e = e0 + (int)threadIdx.x; e < e1; e += kThreads) d[e] = (short)(ci[e] - b);
    }
}

// ---------------------------------------------------------------- sliced-diagonal SpMV
// The sliced-diagonal form of a CSR matrix whose rows, a slice of up to 32 R at a time, share a
// few diagonals (R rows a lane: 1 or 2 for FP64 values, 2 for FP32, 4 for BF16, so that a
// lane's values of one diagonal are one load). Slices never straddle a segment boundary (the
// systems of a batch; one segment for a single system), so a segment's last slice may hold
// fewer rows. Slice s holds its rows' diagonals d = col - row, ascending; each diagonal stores
// one value per row slot of the slice (v[32 R k + row - first row], k counted over all
// slices). A row's own entries keep their storage order (rows are sorted by column), and a
// slot the row has no entry in holds the padding pattern (kDiaPad, kDiaPad32, kDiaPad16: NaN
// bit patterns no entry of the matrix holds, checked when the values are placed). Each slice
// has a record of rs ints (16 or 32): its first diagonal k0, its count m (with kDiaClamp when
// a slot's column falls outside the matrix), its m offsets, and in its last two ints its first
// row and its row count; a warp reads it in one coalesced load. Bytes per entry: the value's
// width and the padding, plus 2 or 4 per R rows for the records, against the width plus 2 or
// 4 per entry and 4 per row for the CSR streams.
constexpr unsigned long long kDiaPad = 0xFFF7D1A6B00C5A1DULL;   // FP64 padding; FP32 and BF16 below
constexpr unsigned kDiaPad32 = 0xFFD1A6B5u;
constexpr unsigned short kDiaPad16 = 0xFFD1u;
constexpr int kDiaRecHead = 2;     // record: k0, count | flags, offsets ..., first row, rows
constexpr int kDiaMaxDiags = 32 - kDiaRecHead - 2;   // diagonals of one slice at most
constexpr int kDiaCountMask = 0xffff, kDiaClamp = 1 << 30;   // record[1]: count | clamp flag

template <typename V = double>
struct DiaView {
    const int *__restrict__ rec;      // nsl records of rs ints: k0, m, first row, rows, offsets
    const V *__restrict__ v;          // 32 R values per diagonal
    int n, nsl, rs;
};

// A lane's R values of one diagonal (one load of R values, streamed) and the padding test;
// BF16 is widened by a shift or a mask, so the padding keeps its pattern in the upper half.
// R is 1 or 2 for FP64, 2 for FP32, 4 for BF16.
template <typename V, int R>
struct DiaLoad;
template <int R>
struct DiaLoad<double, R> {   // the upper word decides: no entry of a served matrix shares it
    using E = double;
    static __device__ __forceinline__ void get(const double *p, double (&a)[R]) {
        if constexpr (R == 2) {
            const double2 w = __ldcs(reinterpret_cast<const double2 *>(p));
            a[0] = w.x;
            a[1] = w.y;
        } else {
            a[0] = ldm(p);
        }
    }
    static __device__ __forceinline__ bool pad(double a) { return __double2hiint(a) == (int)(kDiaPad >> 32); }
};
template <>
struct DiaLoad<float, 2> {
    using E = float;
    static __device__ __forceinline__ void get(const float *p, float (&a)[2]) {
        const float2 w = __ldcs(reinterpret_cast<const float2 *>(p));
        a[0] = w.x;
        a[1] = w.y;
    }
    static __device__ __forceinline__ bool pad(float a) { return __float_as_uint(a) == kDiaPad32; }
};
template <>
struct DiaLoad<__nv_bfloat16, 4> {
    using E = float;
    static __device__ __forceinline__ void get(const __nv_bfloat16 *p, float (&a)[4]) {
        const uint2 w = __ldcs(reinterpret_cast<const uint2 *>(p));
        a[0] = __uint_as_float(w.x << 16);
        a[1] = __uint_as_float(w.x & 0xffff0000u);
        a[2] = __uint_as_float(w.y << 16);
        a[3] = __uint_as_float(w.y & 0xffff0000u);
    }
    static __device__ __forceinline__ bool pad(float a) { return __float_as_uint(a) == ((unsigned)kDiaPad16 << 16); }
};
__device__ __forceinline__ double dia_fma(double s, double a, double x) { return __dadd_rn(s, __dmul_rn(a, x)); }
__device__ __forceinline__ float dia_fma(float s, float a, float x) { return __fadd_rn(s, __fmul_rn(a, x)); }

// A lane's R gathered x of one diagonal d for its rows row0 .. row0 + R - 1 (row0 = the
// slice's first row + R lane, R even when R > 1, so row0 + d has the same parity in every
// lane). A slice whose slots all stay inside the matrix (no kDiaClamp flag) reads without
// clamping, pairs as one load when row0 + d is even (the pair then starts on its own width);
// otherwise each column is clamped to [0, n) (padding slots may point outside; their x is
// never used).
template <bool CLAMP, int R, typename T>
__device__ __forceinline__ void dia_gather(const T *__restrict__ x, int row0, int d, int n, T (&xv)[R]) {
    if constexpr (!CLAMP && R >= 2) {
        if (((row0 + d) & 1) == 0) {
            using T2 = std::conditional_t<sizeof(T) == 8, double2, float2>;
#pragma unroll
            for (int j = 0; j < R; j += 2) {
                const T2 w = __ldg(reinterpret_cast<const T2 *>(x + row0 + d + j));
                xv[j] = w.x;
                xv[j + 1] = w.y;
            }
            return;
        }
    }
#pragma unroll
    for (int j = 0; j < R; ++j) {
        const int c = row0 + j + d;
        xv[j] = ldx(x + (CLAMP ? min(max(c, 0), n - 1) : c));
    }
}

// One warp per slice, R rows a lane, grid-stride; the next slice's record is loaded while the
// current one is summed, and a chunk's value loads and gathers are all issued before any is
// summed. A thread sums each of its rows in storage order exactly as the CSR-stream kernels
// do (from 0, products then sums each rounded, padding skipped), so every form gives the same
// bits. Lanes read consecutive values and, on a banded matrix, consecutive x. Two slices per
// warp trip took about 100 registers a thread and measured slower (H's FP64 product at 128^3:
// 78.9 against 42.9 us). The kernels are bound by instruction issue (63 % issue active at 48 %
// warps active), so with 2 or 4 rows a lane a slice that needs no clamping takes a path
// without it, with paired FP32 gathers; for FP64 that path lost its loads' overlap (long-
// scoreboard stalls 15.4 against 7.2 an issue, H's product 67.0 against 47.7 us under ncu),
// so FP64 always clamps.
// One slice (record rec, its first ints held by lanes 0 .. rs - 1): sums each live row of the
// lane and hands it to emit(row, sum, operand) (operand: the epilogue's pre(row) when it has
// one). Values are loaded in their stored type E and widened to T (FP64 vectors over FP32
// factors in the batched solve) at the product.
template <typename V, typename T, int R, typename Epi, typename Emit>
__device__ __forceinline__ void dia_slice(const DiaView<V> &M, const T *__restrict__ x, const Epi &epi, int rec,
                                          int lane, Emit &&emit) {
    using E = typename DiaLoad<V, R>::E;
    constexpr int SH = 32 * R;
    constexpr int C = 64 / (R * (int)sizeof(E));   // diagonals a chunk: 64 bytes of values a thread
    const unsigned full = 0xffffffffu;
    const int k0 = __shfl_sync(full, rec, 0), mf = __shfl_sync(full, rec, 1);
    const int first = __shfl_sync(full, rec, M.rs - 2), rows = __shfl_sync(full, rec, M.rs - 1);
    const int m = mf & kDiaCountMask;
    const int row0 = first + R * lane;
    T opnd[R], s[R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
        opnd[j] = T(0);
        if constexpr (HasPre<Epi>::value) opnd[j] = R * lane + j < rows ? epi.pre(row0 + j) : T(0);
        s[j] = T(0);
    }
    auto sum = [&](auto clamp) {
        constexpr bool CL = decltype(clamp)::value;
        for (int k = 0; k < m; k += C) {
            E a[C][R];
            T xv[C][R];
#pragma unroll
            for (int u = 0; u < C; ++u) {
                const int d = __shfl_sync(full, rec, (kDiaRecHead + k + u) & 31);
#pragma unroll
                for (int j = 0; j < R; ++j) {
                    a[u][j] = E(0);
                    xv[u][j] = T(0);
                }
                if (k + u < m) {
                    DiaLoad<V, R>::get(M.v + (long)(k0 + k + u) * SH + R * lane, a[u]);
                    dia_gather<CL, R>(x, row0, d, M.n, xv[u]);
                }
            }
#pragma unroll
            for (int u = 0; u < C; ++u)
#pragma unroll
                for (int j = 0; j < R; ++j)
                    if (k + u < m && !DiaLoad<V, R>::pad(a[u][j])) s[j] = dia_fma(s[j], T(a[u][j]), xv[u][j]);
        }
    };
    if (R == 1 || (mf & kDiaClamp)) sum(std::true_type{});
    else sum(std::false_type{});
#pragma unroll
    for (int j = 0; j < R; ++j)
        if (R * lane + j < rows) emit(row0 + j, s[j], opnd[j]);
}

// One warp per slice of a single system (one segment: slice s starts at row 32 R s, so its
// rows follow from s and the matrix's n), grid-stride; the next slice's record is loaded while
// the current one is summed, and a chunk's value loads and gathers are all issued before any
// is summed. A thread sums each of its rows in storage order exactly as the CSR-stream kernels
// do (from 0, products then sums each rounded, padding skipped), so every form gives the same
// bits. Lanes read consecutive values and, on a banded matrix, consecutive x. This body is
// dia_slice's with the slice's rows taken from s: reading them from the record, as dia_slice
// must for the batch's segments, measured 5 % slower on the 128^3 FP64 solve (G's product with
// its norm 28.9 against 24.7 us, A's with omega 30.5 against 27.3 us, the same box).
// Two slices per warp trip took about 100 registers a thread and measured slower (H's FP64
// product at 128^3: 78.9 against 42.9 us). The kernels are bound by instruction issue (63 %
// issue active at 48 % warps active), so with 2 or more rows a lane a slice that needs no
// clamping takes a path without it, gathering pairs as one load; with one row a lane that path
// lost its loads' overlap (long-scoreboard stalls 15.4 against 7.2 an issue, H's product 67.0
// against 47.7 us under ncu), so one row a lane always clamps.
template <typename V, typename T, int R, typename Epi>
static __global__ void __launch_bounds__(kThreads)
k_spmv_dia(DiaView<V> M, const T *__restrict__ x, Epi epi, DState *st, double *__restrict__ partials) {
    static_assert(std::is_same_v<typename DiaLoad<V, R>::E, T>, "one system: values load as T");
    constexpr int SH = 32 * R;
    constexpr int C = 64 / (R * (int)sizeof(T));   // diagonals a chunk: 64 bytes of values a thread
    pdl_enter();
    if (Epi::GATED && st != nullptr && st->done) return;
    double red[Epi::NR];
#pragma unroll
    for (int j = 0; j < Epi::NR; ++j) red[j] = 0.0;
    const int lane = (int)threadIdx.x & 31;
    const int nw = (int)gridDim.x * kWarps;
    const unsigned full = 0xffffffffu;
    int sl = (int)blockIdx.x * kWarps + ((int)threadIdx.x >> 5);
    int rec = (sl < M.nsl && lane < M.rs) ? __ldg(M.rec + (long)sl * M.rs + lane) : 0;
    for (; sl < M.nsl; sl += nw) {
        const int nxt = sl + nw;
        const int rec_next = (nxt < M.nsl && lane < M.rs) ? __ldg(M.rec + (long)nxt * M.rs + lane) : 0;
        const int row0 = sl * SH + R * lane;
        T opnd[R], s[R];
#pragma unroll
        for (int j = 0; j < R; ++j) {
            opnd[j] = T(0);
            if constexpr (HasPre<Epi>::value) opnd[j] = row0 + j < M.n ? epi.pre(row0 + j) : T(0);
            s[j] = T(0);
        }
        const int k0 = __shfl_sync(full, rec, 0), mf = __shfl_sync(full, rec, 1);
        const int m = mf & kDiaCountMask;
        auto sum = [&](auto clamp) {
            constexpr bool CL = decltype(clamp)::value;
            for (int k = 0; k < m; k += C) {
                T a[C][R], xv[C][R];
#pragma unroll
                for (int u = 0; u < C; ++u) {
                    const int d = __shfl_sync(full, rec, (kDiaRecHead + k + u) & 31);
#pragma unroll
                    for (int j = 0; j < R; ++j) {
                        a[u][j] = T(0);
                        xv[u][j] = T(0);
                    }
                    if (k + u < m) {
                        DiaLoad<V, R>::get(M.v + (long)(k0 + k + u) * SH + R * lane, a[u]);
                        dia_gather<CL, R>(x, row0, d, M.n, xv[u]);
                    }
                }
#pragma unroll
                for (int u = 0; u < C; ++u)
#pragma unroll
                    for (int j = 0; j < R; ++j)
                        if (k + u < m && !DiaLoad<V, R>::pad(a[u][j])) s[j] = dia_fma(s[j], a[u][j], xv[u][j]);
            }
        };
        if (R == 1 || (mf & kDiaClamp)) sum(std::true_type{});
        else sum(std::false_type{});
#pragma unroll
        for (int j = 0; j < R; ++j) {
            if (row0 + j < M.n) {
                if constexpr (HasPre<Epi>::value) epi.emit_pre(row0 + j, s[j], opnd[j], red);
                else epi.emit(row0 + j, s[j], red);
            }
        }
        rec = rec_next;
    }
    pdl_release();
    if constexpr (Epi::REDUCES) grid_reduce<Epi::NR>(red, partials, st, epi);
}

// ---------------------------------------------------------------- CSR-vector SpMV
// For callers without set-up (the kernel-level C-ABI): VEC lanes per row, 32/VEC rows
// per warp, grid-stride over row groups. Each lane rounds its product; the group then
// adds the products in storage order by broadcasting them lane by lane, so the sum is
// the same as the left-to-right CSR loop for every VEC. FILL 0 uses every entry; 1
// keeps col >= row and 2 keeps col <= row (MKL's TRIANGULAR descriptors).
template <int VEC, typename Epi, int FILL = 0>
static __global__ void __launch_bounds__(kThreads)
k_spmv_vec(CsrView<double> M, const double *__restrict__ x, Epi epi, DState *st,
           double *__restrict__ partials) {
    if (Epi::GATED && st != nullptr && st->done) return;
    constexpr int RPW = 32 / VEC;
    const int lane = threadIdx.x & 31;
    const int sub = lane / VEC, lir = lane % VEC, gbase = sub * VEC;
    const long warp = ((long)blockIdx.x * kThreads + threadIdx.x) >> 5;
    const long nwarps = ((long)gridDim.x * kThreads) >> 5;
    double red[Epi::NR];
#pragma unroll
    for (int j = 0; j < Epi::NR; ++j) red[j] = 0.0;
    for (long base = warp * RPW; base < M.n; base += nwarps * RPW) {
        const long row = base + sub;
        int beg = 0, len = 0;
        if (row < M.n) {
            beg = __ldg(M.rp + row);
            len = __ldg(M.rp + row + 1) - beg;
        }
        const int trips = __reduce_max_sync(0xffffffffu, (len + VEC - 1) / VEC);
        double s = 0.0;
        for (int t = 0; t < trips; ++t) {
            const int k = t * VEC + lir;
            double p = 0.0;
            int keep = 0;
            if (k < len) {
                const int c = ldi(M.ci + beg + k);
                keep = !((FILL == 1 && c < row) || (FILL == 2 && c > row));
                if (keep) p = __dmul_rn(ldm(M.v + beg + k), ldx(x + c));
            }
#pragma unroll
            for (int j = 0; j < VEC; ++j) {
                const double pj = __shfl_sync(0xffffffffu, p, gbase + j);
                const int kj = __shfl_sync(0xffffffffu, keep, gbase + j);
                if (kj) s = __dadd_rn(s, pj);
            }
        }
        if (row < M.n && lir == 0) epi.emit(row, s, red);
    }
    if constexpr (Epi::REDUCES) grid_reduce<Epi::NR>(red, partials, st, epi);
}

// ---------------------------------------------------------------- streaming kernels
// Grid-stride loop shared by the elementwise kernels.
#define FIIM_FOR_ROWS(i, n) \
    for (long i = (long)blockIdx.x * kThreads + threadIdx.x; i < (n); i += (long)gridDim.x * kThreads)

// Grid-stride loop over [0, n), U elements per trip: the loads of all U elements (ld(i)
// returns them as one value) are issued before any is used (op(i, loaded)), so a thread has
// U times as many loads in flight. A thread still visits its elements in ascending order, so
// its partial sums are those of the plain loop, bit for bit.
template <int U, class Ld, class Op>
__device__ __forceinline__ void stream_rows(long n, const Ld &ld, const Op &op) {
    const long S = (long)gridDim.x * kThreads;
    long i = (long)blockIdx.x * kThreads + threadIdx.x;
    for (; i + (U - 1) * S < n; i += U * S) {
        decltype(ld(0L)) q[U];
#pragma unroll
        for (int u = 0; u < U; ++u) q[u] = ld(i + u * S);
#pragma unroll
        for (int u = 0; u < U; ++u) op(i + u * S, q[u]);
    }
    for (; i < n; i += S) op(i, ld(i));
}

struct Ld3 {
    double a, b, c;
};
struct Ld6 {
    double a, b, c, d, e, f;
};

struct FinS {
    __device__ void finish(DState *st, const double *t) const {
        st->r2 = t[0];
        st->x2 = t[1];
    }
};

// s = r + (-alpha) v (cblas_dcopy + cblas_daxpy, AFIIM/src/bicgstab.cpp:184-185);
// ||r||^2 (the residual norm the reference tests, taken before r is updated, :216)
// and ||x||^2 (stagnation test, :201). Fin receives the two sums (FinS stores them in the
// scalars; a row-partitioned solve exports its block's sums instead).
template <class Fin>
static __global__ void __launch_bounds__(kThreads)
k_update_s(long n, const double *__restrict__ r, const double *__restrict__ v,
           const double *__restrict__ x, double *__restrict__ s, DState *st,
           double *__restrict__ partials, Fin fin) {
    pdl_enter();
    if (st->done) return;
    const double na = -st->alpha;
    double red[2] = {0.0, 0.0};
    stream_rows<1>(   // unrolling measured slower here (12.2 against 10.7 us at 128^3)
        n, [&](long i) { return Ld3{r[i], v[i], x[i]}; },
        [&](long i, const Ld3 &q) {
            s[i] = __dadd_rn(q.a, __dmul_rn(na, q.b));
            red[0] += q.a * q.a;
            red[1] += q.c * q.c;
        });
    pdl_release();
    grid_reduce<2>(red, partials, st, fin);
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

// x = x + alpha pc; x = x + omega sc; r = s + (-omega) t (AFIIM/src/bicgstab.cpp:207-259);
// sum r0 . r; then the tests (Fin = FinControl; a row-partitioned solve exports the sum).
template <class Fin>
static __global__ void __launch_bounds__(kThreads)
k_update_xr(long n, const double *__restrict__ pc, const double *__restrict__ sc,
            const double *__restrict__ s, const double *__restrict__ t,
            const double *__restrict__ r0, double *__restrict__ x, double *__restrict__ r,
            DState *st, double *__restrict__ partials, Fin fin) {
    pdl_enter();
    if (st->done) return;
    const double a = st->alpha, om = st->omega, nom = -st->omega;
    double red[1] = {0.0};
    stream_rows<4>(   // 26.0 against 27.6 us at 128^3
        n, [&](long i) { return Ld6{x[i], pc[i], sc[i], s[i], t[i], r0[i]}; },
        [&](long i, const Ld6 &q) {
            double xi = q.a;
            xi = __dadd_rn(xi, __dmul_rn(a, q.b));
            xi = __dadd_rn(xi, __dmul_rn(om, q.c));
            x[i] = xi;
            const double ri = __dadd_rn(q.d, __dmul_rn(nom, q.e));
            r[i] = ri;
            red[0] += q.f * ri;
        });
    pdl_release();
    grid_reduce<1>(red, partials, st, fin);
}

// p = (-beta omega) v + beta p; p = p + r (cblas_daxpby + cblas_daxpy,
// AFIIM/src/bicgstab.cpp:270-271). In the device-driven loop this is the last kernel of
// the body: block 0 counts the body, trips a guard (info -5) should the body ever run
// past nmax + 2 times, and sets the WHILE node's condition to continue only while the
// solve is not done.
static __global__ void __launch_bounds__(kThreads)
k_update_p(long n, const double *__restrict__ r, const double *__restrict__ v,
           double *__restrict__ p, DState *st, cudaGraphConditionalHandle h, int cond) {
    pdl_enter();
    if (cond && blockIdx.x == 0 && threadIdx.x == 0) {
        const int loops = ++st->loops;
        if (!st->done && loops > st->nmax + 2) {
            st->info = -5;
            st->done = 1;
        }
        cudaGraphSetConditional(h, st->done ? 0u : 1u);
    }
    if (st->done) return;
    const double b = st->beta, c = __dmul_rn(-st->beta, st->omega);
    stream_rows<4>(
        n, [&](long i) { return Ld3{v[i], p[i], r[i]}; },
        [&](long i, const Ld3 &q) { p[i] = __dadd_rn(__dadd_rn(__dmul_rn(c, q.a), __dmul_rn(b, q.b)), q.c); });
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

// Sliced-diagonal values, moved as bit patterns B of the value's width (8, 4 or 2 bytes):
// every slot padding, then each entry e to its slot map[e]; *bad is set when an entry holds
// the padding's pattern.
template <typename B>
static __global__ void __launch_bounds__(kThreads)
k_dia_fill(long slots, B *__restrict__ dv, B pad) {
    FIIM_FOR_ROWS(i, slots) { dv[i] = pad; }
}
template <typename B>
__device__ __forceinline__ bool dia_is_pad(B o, B pad) {   // the kernel's test (upper word of FP64)
    if constexpr (sizeof(B) == 8) return (o >> 32) == (pad >> 32);
    else return o == pad;
}
template <typename B>
static __global__ void __launch_bounds__(kThreads)
k_dia_scatter(long nnz, const B *__restrict__ v, const int *__restrict__ map, B *__restrict__ dv, B pad, int *bad) {
    FIIM_FOR_ROWS(e, nnz) {
        const B o = v[e];
        if (dia_is_pad(o, pad)) atomicExch(bad, 1);
        dv[map[e]] = o;
    }
}

// Whether new column indices (with unchanged row offsets) still fit the slices' diagonals:
// entry e of row i of a slice must sit in slot map[e] = sh k + i - first of a diagonal k of
// the slice (k0 <= k < k0 + m) whose offset is ci[e] - i; sh = 32 R row slots a slice. *bad
// is set otherwise. One warp per slice, its lanes over the slice's rows.
static __global__ void __launch_bounds__(kThreads)
k_dia_check(int nsl, const int *__restrict__ rp, const int *__restrict__ ci, const int *__restrict__ map,
            const int *__restrict__ rec, int rs, int sh, int *bad) {
    const int lane = (int)threadIdx.x & 31;
    for (int sl = (int)blockIdx.x * kWarps + ((int)threadIdx.x >> 5); sl < nsl; sl += (int)gridDim.x * kWarps) {
        const int *r = rec + (long)sl * rs;
        const int k0 = r[0], m = r[1] & kDiaCountMask, first = r[rs - 2], rows = r[rs - 1];
        for (int t = lane; t < rows; t += 32) {
            const int i = first + t;
            for (int e = rp[i]; e < rp[i + 1]; ++e) {
                const int slot = map[e], k = slot / sh - k0;
                if (slot % sh != t || k < 0 || k >= m || r[kDiaRecHead + k] != ci[e] - i) {
                    atomicExch(bad, 1);
                    break;
                }
            }
        }
    }
}

// Order-sensitive hash of a column stream: the wrapping sum over entries of the splitmix64
// finalizer (Steele, Lea and Flood, OOPSLA 2014) of (position, column), so the sum's order
// does not matter. Tells whether a matrix's columns changed since a set-up decision.
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
static __global__ void __launch_bounds__(kThreads)
k_col_hash(long nnz, const int *__restrict__ ci, unsigned long long *out) {
    unsigned long long h = 0;
    FIIM_FOR_ROWS(e, nnz) { h += mix64(((unsigned long long)e << 32) | (unsigned)ci[e]); }
    for (int o = 16; o > 0; o >>= 1) h += __shfl_down_sync(0xffffffffu, h, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, h);
}

}  // namespace fiim
