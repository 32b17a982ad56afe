// Device kernels of the batched solve: many independent systems, concatenated as one
// block-diagonal CSR, each running the reference's BiCGSTAB (AFIIM/src/bicgstab.cpp:168-275
// or ACIFIM/src/bicgstab.cpp:197-304) with its own scalars and termination.
//
// Row blocks (<= 256 rows, <= TILE - 1 entries) never straddle two systems. Every kernel walks
// row blocks; a block of a system that has finished is skipped. Reductions are per system:
// each warp of each row block stores one partial, and a finish kernel (one CTA per system)
// adds a system's partials in a fixed order and applies the system's scalar step. Vectors
// are FP64; factor values may be FP64, FP32 or BF16 (widened to FP64 before the rounded
// product), so every vector operation is the reference's, bit for bit,
// on the factors as stored.
#pragma once

#include "fiim_kernels.cuh"

namespace fiim {
namespace bt {

struct BGlobal {
    double tol, eps;
    int nmax, alpha_guard, active, loops;
    int loops_total;   // verified solves: loop bodies of the runs before the current one
};

// Finished-system flags per row block (or per slice of a sliced-diagonal copy) of one matrix
// (batched solve; NULL elsewhere): flag[b] != 0 once the system of block b has left the loop,
// so a kernel can skip a block with one load that needs no other.
struct BlockFlags {
    int *flag;
    const int *sys_blk;   // nsys + 1 block offsets per system
};

// Per-system state, structure of arrays (nsys entries each).
struct BState {
    double *ro, *rc, *m1, *m2, *alpha, *omega, *beta, *pc2, *x2, *r2, *ts, *tt;
    int *iter, *stag, *msteps, *maxmsteps, *info, *done;
    unsigned int *ticket;   // per-system tickets (the block solver's last-CTA reductions)
    BGlobal *g;
    BlockFlags bf[6];       // A, G, H row blocks, then the slices of their sliced-diagonal copies
};

// A system leaves the loop. Its row-block and slice flags are then set by the whole CTA of
// the finish kernel that retired it (k_bfinish): a large system has thousands of slices, and
// one thread setting them all cost up to ~45 us a launch.
__device__ __forceinline__ void retire(BState &bs, int k, int info) {
    bs.info[k] = info;
    bs.done[k] = 1;
    atomicSub(&bs.g->active, 1);
}

// ---------------------------------------------------------------- per-system scalar steps
struct BFinInit {   // ro = ||r0||, m1 = ro^2, rc = ro (AFIIM/src/bicgstab.cpp:161-165)
    __device__ void finish(BState &bs, int k, const double *t) const {
        bs.ro[k] = sqrt(t[0]);
        bs.m1[k] = bs.ro[k] * bs.ro[k];
        bs.rc[k] = bs.ro[k];
        bs.iter[k] = 0;
        bs.stag[k] = 0;
        bs.msteps[k] = 0;
        if (bs.g->nmax <= 0) retire(bs, k, bs.g->nmax == 0 ? 3 : -1);
    }
};
// Verified solves: a system re-enters the loop from its current x. As at the start,
// r = r0 = p = b - A x and rc = ||r||, m1 = rc^2 (AFIIM/src/bicgstab.cpp:161-165), and the
// stagnation and divergence counters restart; ro (the test's reference norm, ||b - A x0||)
// and the iteration count carry on.
struct BFinRestart {
    __device__ void finish(BState &bs, int k, const double *t) const {
        bs.rc[k] = sqrt(t[0]);
        bs.m1[k] = bs.rc[k] * bs.rc[k];
        bs.stag[k] = 0;
        bs.msteps[k] = 0;
    }
};

// Verified solves: the FP64 true residual ||b - A x|| (ts, from BEpiResid) of a system that
// left the loop converged (info 0) must be below tol * ro, the reference's test applied to
// the true residual in place of the recurrence one. A system that misses it is marked
// running again (its row blocks unflagged) and counted in active; the runs' loop counts are
// folded into loops_total.
__device__ __forceinline__ bool verify_misses(const BState &bs, int k) {
    if (bs.info[k] != 0 || bs.ts[k] == 0.0) return false;
    return !(sqrt(bs.ts[k]) < bs.g->tol * bs.ro[k]);
}

static __global__ void __launch_bounds__(kThreads) k_bverify(int nsys, BState bs) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        bs.g->loops_total += bs.g->loops;
        bs.g->loops = 0;
    }
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nsys; k += gridDim.x * blockDim.x) {
        if (!verify_misses(bs, k)) continue;
        bs.done[k] = 0;
        bs.info[k] = -1;
        for (int m = 0; m < 6; ++m)
            if (bs.bf[m].flag)
                for (int b = bs.bf[m].sys_blk[k]; b < bs.bf[m].sys_blk[k + 1]; ++b) bs.bf[m].flag[b] = 0;
        atomicAdd(&bs.g->active, 1);
    }
}

struct BFinS {
    __device__ void finish(BState &bs, int k, const double *t) const {
        bs.r2[k] = t[0];
        bs.x2[k] = t[1];
    }
};
struct BFinControl {   // AFIIM/src/bicgstab.cpp:201-274, per system
    __device__ void finish(BState &bs, int k, const double *t) const {
        const double a = bs.alpha[k], om = bs.omega[k];
        if (fabs(a) * sqrt(bs.pc2[k]) < bs.g->eps * sqrt(bs.x2[k])) bs.stag[k]++;
        else bs.stag[k] = 0;
        const double prc = bs.rc[k];
        bs.rc[k] = sqrt(bs.r2[k]);
        if (prc < bs.rc[k]) bs.msteps[k]++;
        else bs.msteps[k] = 0;
        if (bs.msteps[k] >= bs.maxmsteps[k]) { retire(bs, k, 1); return; }
        if (bs.stag[k] >= 3) { retire(bs, k, 2); return; }
        if (bs.rc[k] < bs.g->tol * bs.ro[k]) { retire(bs, k, 0); return; }
        bs.m2[k] = bs.m1[k];
        bs.m1[k] = t[0];
        bs.beta[k] = bs.m1[k] * a / (om * bs.m2[k]);
        bs.iter[k]++;
        if (bs.iter[k] >= bs.g->nmax) retire(bs, k, 3);
    }
};

// ---------------------------------------------------------------- epilogues (FP64 vectors)
struct BEpiScale {
    FIIM_EPI(1, false, true);
    double *y;
    const double *__restrict__ d;
    __device__ double pre(long i) const { return __ldg(d + i); }
    __device__ void emit_pre(long i, double s, double di, double (&)[NR]) const { y[i] = __dmul_rn(di, s); }
    __device__ void emit(long i, double s, double (&r)[NR]) const { emit_pre(i, s, pre(i), r); }
    __device__ void finish(BState &, int, const double *) const {}
};
struct BEpiStore {
    FIIM_EPI(1, false, true);
    double *y;
    __device__ void emit(long i, double s, double (&)[NR]) const { y[i] = s; }
    __device__ void finish(BState &, int, const double *) const {}
};
struct BEpiNorm {
    FIIM_EPI(1, true, true);
    double *y;
    __device__ void emit(long i, double s, double (&r)[NR]) const { y[i] = s; r[0] += s * s; }
    __device__ void finish(BState &bs, int k, const double *t) const { bs.pc2[k] = t[0]; }
};
struct BEpiAlpha {
    FIIM_EPI(1, true, true);
    double *y;
    const double *__restrict__ r0;
    __device__ double pre(long i) const { return __ldg(r0 + i); }
    __device__ void emit_pre(long i, double s, double r0i, double (&r)[NR]) const {
        y[i] = s;
        r[0] += r0i * s;
    }
    __device__ void emit(long i, double s, double (&r)[NR]) const { emit_pre(i, s, pre(i), r); }
    __device__ void finish(BState &bs, int k, const double *t) const {
        bs.alpha[k] = bs.m1[k] / t[0];
        if (bs.g->alpha_guard && !isfinite(bs.alpha[k])) {   // ACIFIM/src/bicgstab.cpp:208-213
            bs.iter[k] = bs.g->nmax;
            retire(bs, k, 3);
        }
    }
};
struct BEpiOmega {
    FIIM_EPI(2, true, true);
    double *y;
    const double *__restrict__ sv;
    __device__ double pre(long i) const { return __ldg(sv + i); }
    __device__ void emit_pre(long i, double s, double si, double (&r)[NR]) const {
        y[i] = s;
        r[0] += s * si;
        r[1] += s * s;
    }
    __device__ void emit(long i, double s, double (&r)[NR]) const { emit_pre(i, s, pre(i), r); }
    __device__ void finish(BState &bs, int k, const double *t) const { bs.omega[k] = t[0] / t[1]; }
};
struct BEpiInit {
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
    __device__ void finish(BState &bs, int k, const double *t) const { BFinInit{}.finish(bs, k, t); }
};
struct BEpiRestart : BEpiInit {
    __device__ void finish(BState &bs, int k, const double *t) const { BFinRestart{}.finish(bs, k, t); }
};
struct BEpiResid {
    FIIM_EPI(2, true, false);
    const double *__restrict__ b;
    __device__ void emit(long i, double s, double (&red)[NR]) const {
        const double bi = b[i], ri = bi - s;
        red[0] += ri * ri;
        red[1] += bi * bi;
    }
    __device__ void finish(BState &bs, int k, const double *t) const {
        bs.ts[k] = t[0];
        bs.tt[k] = t[1];
    }
};

// ---------------------------------------------------------------- per-system reduction
// Two phases. In a reducing kernel every warp of every row block stores its partial (lane 0,
// after the warp's shuffle tree): no CTA barrier, fence or atomic per block. A finish kernel
// then gives each system one warp, which adds the system's partials (blocks in order,
// lane-strided, then the shuffle tree: a fixed order) and applies the system's scalar step.
// Partials: (block * kWarps + warp) * NR + j. The finish kernel gives each system one CTA.
template <int NR>
__device__ __forceinline__ void warp_partials(double (&v)[NR], int blk, double *__restrict__ partials) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < NR; ++j) v[j] = warp_sum(v[j]);
    if (lane == 0)
#pragma unroll
        for (int j = 0; j < NR; ++j) partials[((size_t)blk * kWarps + w) * NR + j] = v[j];
}

// One CTA per system (grid-stride over systems): thread t adds partials t, t + 256, ...
// of the system, then the CTA's warp trees and the warp totals in warp order (a fixed
// order). Systems whose loop has ended are left alone when GATED. A system's partials are
// [sys_blk[k] qmul, sys_blk[k + 1] qmul): qmul = kWarps for row-block partials (one per warp
// of a block), 1 for slice partials (one per slice).
template <int NR, bool GATED, class Fin>
static __global__ void __launch_bounds__(kThreads)
k_bfinish(const int *__restrict__ sys_blk, int qmul, int nsys, const double *__restrict__ partials, BState bs,
          Fin fin) {
    pdl_enter();
    __shared__ double sm[kWarps][NR];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int k = blockIdx.x; k < nsys; k += gridDim.x) {
        if (GATED && bs.done[k]) continue;             // uniform in the CTA
        const int q0 = __ldg(sys_blk + k) * qmul, q1 = __ldg(sys_blk + k + 1) * qmul;
        double acc[NR];
#pragma unroll
        for (int j = 0; j < NR; ++j) acc[j] = 0.0;
        for (int q = q0 + (int)threadIdx.x; q < q1; q += kThreads)
#pragma unroll
            for (int j = 0; j < NR; ++j) acc[j] += partials[(size_t)q * NR + j];
#pragma unroll
        for (int j = 0; j < NR; ++j) acc[j] = warp_sum(acc[j]);
        if (lane == 0)
#pragma unroll
            for (int j = 0; j < NR; ++j) sm[w][j] = acc[j];
        __syncthreads();
        if (threadIdx.x == 0) {
            double tot[NR];
#pragma unroll
            for (int j = 0; j < NR; ++j) {
                double t = 0.0;
#pragma unroll
                for (int q = 0; q < kWarps; ++q) t += sm[q][j];
                tot[j] = t;
            }
            fin.finish(bs, k, tot);
        }
        __syncthreads();
        if (GATED && bs.done[k])   // retired just now (a finished system was skipped above)
            for (int m = 0; m < 6; ++m)
                if (bs.bf[m].flag)
                    for (int b = bs.bf[m].sys_blk[k] + (int)threadIdx.x; b < bs.bf[m].sys_blk[k + 1]; b += kThreads)
                        bs.bf[m].flag[b] = 1;
    }
}

__device__ __forceinline__ double widen(double v) { return v; }
__device__ __forceinline__ double widen(float v) { return (double)v; }

// ---------------------------------------------------------------- batched CSR-stream SpMV
// The single-system kernel's structure (k_spmv_rows): row blocks of at most TILE - 1
// entries (first rows rb, first entries eb), entries read in aligned pairs, and the loop
// pipelined by one block. The next block's system, bounds, row offsets, entry streams and
// epilogue operand are loaded into registers before the barrier. A block whose system has
// finished loads nothing and is skipped: a system's done flag changes only after all of its
// blocks in the launch have been reduced, so the value read at prefetch is the one at use.
template <int TILE, typename V, typename Epi, bool NARROW = false>
static __global__ void __launch_bounds__(kThreads, 4)
k_bspmv(CsrView<V> M, const int *__restrict__ rb, const int *__restrict__ eb, const int *__restrict__ bflag,
        int nblk, const double *__restrict__ x, Epi epi, BState bs, double *__restrict__ partials,
        NarrowCols nc = NarrowCols{}) {
    pdl_enter();
    __shared__ double prod[TILE];
    constexpr int PER = TILE / kThreads;
    const int tid = (int)threadIdx.x;
    int r0 = 0, r1 = 0, e0 = 0, e1 = 0, rbeg = 0, rend = 0, cbase = 0;
    bool skip = false;
    double opnd = 0.0;
    using VP = ValPair<V>;
    ColRegs<NARROW, PER> c;
    typename VP::T a[PER / 2];
    auto fetch = [&](int blk) {
        r0 = __ldg(rb + blk);
        r1 = __ldg(rb + blk + 1);
        e0 = __ldg(eb + blk);
        e1 = __ldg(eb + blk + 1);
        skip = Epi::GATED && bflag[blk];   // flags change only in the finish kernels
        if (skip) return;
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
                a[u] = VP::zero();
                if (e + 1 < e1) {
                    c.load2(M.ci, nc, e, u);
                    a[u] = VP::load2(M.v + e);
                } else if (e < e1) {
                    c.load1(M.ci, nc, e, u);
                    a[u] = VP::load1(M.v + e);
                }
            }
        }
    };
    if ((int)blockIdx.x < nblk) fetch(blockIdx.x);
    for (int blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
        const int nxt = blk + (int)gridDim.x;
        const int cr0 = r0, cr1 = r1, ce0 = e0, ce1 = e1, cb = rbeg - e0, ce = rend - e0, cbs = cbase;
        const double copnd = opnd;
        if (skip) {                                         // uniform in the CTA
            if (nxt < nblk) fetch(nxt);
            continue;
        }
        double red[Epi::NR];
#pragma unroll
        for (int j = 0; j < Epi::NR; ++j) red[j] = 0.0;
        if (ce1 - ce0 < TILE) {
            const int a0 = ce0 & ~1;
#pragma unroll
            for (int u = 0; u < PER; ++u) {
                const int e = a0 + 2 * (tid + (u >> 1) * kThreads) + (u & 1);
                if (e >= ce0 && e < ce1)
                    prod[e - ce0] = __dmul_rn(widen(VP::get(a[u >> 1], u & 1)), ldx(x + c.get(u, cbs)));
            }
            if (nxt < nblk) fetch(nxt);
            __syncthreads();
            if (cr0 + tid < cr1) {
                double s = 0.0;
                for (int q = cb; q < ce; ++q) s = __dadd_rn(s, prod[q]);
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
                    prod[e - c0] = __dmul_rn(widen(ldm(M.v + e)), ldx(x + j));
                }
                __syncthreads();
                if (tid == 0)
                    for (int q = 0; q < c1 - c0; ++q) s = __dadd_rn(s, prod[q]);
                __syncthreads();
            }
            if (tid == 0) epi.emit(cr0, s, red);
            if (nxt < nblk) fetch(nxt);
        }
        if constexpr (Epi::REDUCES) warp_partials<Epi::NR>(red, blk, partials);
    }
    pdl_release();
}

// ---------------------------------------------------------------- batched sliced-diagonal SpMV
// The single-system kernel's slices (dia_slice in fiim_kernels.cuh), which never straddle two
// systems: one warp per slice, grid-stride, a finished system's slices skipped (sflag, set with
// the system's done flag), and each slice's reductions stored as one partial (lane 0, after
// the warp's tree) for the per-system finish (qmul = 1). Factor values stored in FP32 or BF16
// are widened to FP64 at the rounded product, as in k_bspmv.
template <typename V, int R, typename Epi>
static __global__ void __launch_bounds__(kThreads)
k_bspmv_dia(DiaView<V> M, const int *__restrict__ sflag, const double *__restrict__ x, Epi epi, BState bs,
            double *__restrict__ partials) {
    pdl_enter();
    const int lane = (int)threadIdx.x & 31;
    const int nw = (int)gridDim.x * kWarps;
    int sl = (int)blockIdx.x * kWarps + ((int)threadIdx.x >> 5);
    int rec = (sl < M.nsl && lane < M.rs) ? __ldg(M.rec + (long)sl * M.rs + lane) : 0;
    for (; sl < M.nsl; sl += nw) {
        const int nxt = sl + nw;
        const int rec_next = (nxt < M.nsl && lane < M.rs) ? __ldg(M.rec + (long)nxt * M.rs + lane) : 0;
        if (!(Epi::GATED && sflag[sl])) {   // uniform in the warp
            double red[Epi::NR];
#pragma unroll
            for (int j = 0; j < Epi::NR; ++j) red[j] = 0.0;
            dia_slice<V, double, R>(M, x, epi, rec, lane, [&](int row, double s, double opnd) {
                if constexpr (HasPre<Epi>::value) epi.emit_pre(row, s, opnd, red);
                else epi.emit(row, s, red);
            });
            if constexpr (Epi::REDUCES) {
#pragma unroll
                for (int j = 0; j < Epi::NR; ++j) red[j] = warp_sum(red[j]);
                if (lane == 0)
#pragma unroll
                    for (int j = 0; j < Epi::NR; ++j) partials[(size_t)sl * Epi::NR + j] = red[j];
            }
        }
        rec = rec_next;
    }
    pdl_release();
}

// ---------------------------------------------------------------- batched vector updates
// Each walks A's row blocks (<= 256 rows each); thread t owns row rb[blk] + t.
static __global__ void __launch_bounds__(kThreads)
k_bupdate_s(const int *__restrict__ rb, const int *__restrict__ blk_sys, const int *__restrict__ sys_blk,
            int nblk, const double *__restrict__ r, const double *__restrict__ v,
            const double *__restrict__ x, double *__restrict__ s, BState bs, double *__restrict__ partials) {
    pdl_enter();
    for (int blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
        if (bs.bf[0].flag[blk]) continue;                 // uniform in the CTA
        const int k = __ldg(blk_sys + blk);
        const int row = __ldg(rb + blk) + (int)threadIdx.x;
        double red[2] = {0.0, 0.0};
        if (row < __ldg(rb + blk + 1)) {
            const double ri = r[row], xi = x[row];
            s[row] = __dadd_rn(ri, __dmul_rn(-bs.alpha[k], v[row]));
            red[0] = ri * ri;
            red[1] = xi * xi;
        }
        warp_partials<2>(red, blk, partials);
    }
    pdl_release();
}

static __global__ void __launch_bounds__(kThreads)
k_bupdate_xr(const int *__restrict__ rb, const int *__restrict__ blk_sys, const int *__restrict__ sys_blk,
             int nblk, const double *__restrict__ pc, const double *__restrict__ sc,
             const double *__restrict__ s, const double *__restrict__ t, const double *__restrict__ r0,
             double *__restrict__ x, double *__restrict__ r, BState bs, double *__restrict__ partials) {
    pdl_enter();
    for (int blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
        if (bs.bf[0].flag[blk]) continue;
        const int k = __ldg(blk_sys + blk);
        const int row = __ldg(rb + blk) + (int)threadIdx.x;
        double red[1] = {0.0};
        if (row < __ldg(rb + blk + 1)) {
            const double a = bs.alpha[k], om = bs.omega[k];
            double xi = x[row];
            xi = __dadd_rn(xi, __dmul_rn(a, pc[row]));
            xi = __dadd_rn(xi, __dmul_rn(om, sc[row]));
            x[row] = xi;
            const double ri = __dadd_rn(s[row], __dmul_rn(-om, t[row]));
            r[row] = ri;
            red[0] = r0[row] * ri;
        }
        warp_partials<1>(red, blk, partials);
    }
    pdl_release();
}

// Last kernel of the loop body: block 0 counts the body, stops the loop should it ever run
// past nmax + 2 times (active = -1 flags that), and keeps the WHILE node going while any
// system is active.
static __global__ void __launch_bounds__(kThreads)
k_bupdate_p(const int *__restrict__ rb, const int *__restrict__ blk_sys, int nblk,
            const double *__restrict__ r, const double *__restrict__ v, double *__restrict__ p, BState bs,
            cudaGraphConditionalHandle h, int cond) {
    pdl_enter();
    if (cond && blockIdx.x == 0 && threadIdx.x == 0) {
        const int loops = ++bs.g->loops;
        if (bs.g->active > 0 && loops > bs.g->nmax + 2) bs.g->active = -1;
        cudaGraphSetConditional(h, bs.g->active > 0 ? 1u : 0u);
    }
    for (int blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
        if (bs.bf[0].flag[blk]) continue;
        const int k = __ldg(blk_sys + blk);
        const int row = __ldg(rb + blk) + (int)threadIdx.x;
        if (row >= __ldg(rb + blk + 1)) continue;
        const double b = bs.beta[k], c = __dmul_rn(-bs.beta[k], bs.omega[k]);
        const double pi = __dadd_rn(__dmul_rn(c, v[row]), __dmul_rn(b, p[row]));
        p[row] = __dadd_rn(pi, r[row]);
    }
    pdl_release();
}

// Factor values to FP32 / BF16 (round to nearest) for the reduced-precision factor forms.
static __global__ void __launch_bounds__(kThreads)
k_vals_to_f32(long n, const double *__restrict__ in, float *__restrict__ out) {
    FIIM_FOR_ROWS(i, n) { out[i] = __double2float_rn(in[i]); }
}

}  // namespace bt
}  // namespace fiim
