// Device kernels of the multi-RHS block solve: k <= 32 right-hand sides of one system,
// each running the reference's BiCGSTAB (AFIIM/src/bicgstab.cpp:168-275) with its own
// scalars and termination, sharing every sparse product.
//
// Vectors are n x k, row-major (entry (i, j) at i*k + j), so the k values a gathered
// column index needs are contiguous. Work mapping: a lane group of L lanes (a power of two)
// takes one row and each lane owns VW consecutive right-hand sides (lane l: columns l*VW ..
// l*VW + VW - 1; VW = 1, 2 or 4, loaded as one or two 16-byte pairs); a warp holds 32/L row
// groups; warps walk rows in grid-stride order. The vector updates use VW = 1 and
// L = next power of two >= k; the sparse products take their (L, VW) from the solver's shape
// (the row groups per warp and the load width), which never changes a product.
// Sparse products: the group loads the row's entries L at a time (coalesced) and
// broadcasts them lane by lane, so each right-hand side's row sum is formed left to right
// in storage order with rounded products (the reference's arithmetic, bit for bit).
// Reductions are per right-hand side: lanes of equal j are combined within the warp and
// the CTA in a fixed tree, the CTA writes k partials, and the last CTA (ticket) adds them
// in CTA order and runs each right-hand side's scalar step.
#pragma once

#include "fiim_batch.cuh"
#include "fiim_kernels.cuh"

namespace fiim {
namespace bk {

using bt::BState;

struct Shape {
    long n;
    int k;        // right-hand sides
};

// Per-RHS reduction over the CTA and the grid; every thread calls it (uniformly). A thread
// holds the partials of its VW right-hand sides (lane % L) * VW + u, u < VW.
template <int L, int VW, int NR, class Fin>
__device__ __forceinline__ void rhs_reduce(double (&v)[VW][NR], int k, double *__restrict__ partials, BState &bs,
                                           const Fin &fin) {
    __shared__ double sm[kWarps][32][NR];
    __shared__ int last;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    // combine the row groups of the warp (lanes with the same right-hand sides)
#pragma unroll
    for (int u = 0; u < VW; ++u)
#pragma unroll
        for (int j = 0; j < NR; ++j)
#pragma unroll
            for (int o = L; o < 32; o <<= 1) v[u][j] += __shfl_xor_sync(0xffffffffu, v[u][j], o);
    if (lane < L)
#pragma unroll
        for (int u = 0; u < VW; ++u)
#pragma unroll
            for (int j = 0; j < NR; ++j) sm[w][lane * VW + u][j] = v[u][j];
    __syncthreads();
    if (threadIdx.x < k) {
        const int jj = threadIdx.x;
#pragma unroll
        for (int j = 0; j < NR; ++j) {
            double s = 0.0;
#pragma unroll
            for (int q = 0; q < kWarps; ++q) s += sm[q][jj][j];
            partials[((size_t)blockIdx.x * 32 + jj) * NR + j] = s;
        }
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned t = atomicAdd(bs.ticket, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (threadIdx.x < k) {
        const int jj = threadIdx.x;
        double tot[NR];
#pragma unroll
        for (int j = 0; j < NR; ++j) tot[j] = 0.0;
        for (int c = 0; c < (int)gridDim.x; ++c)
#pragma unroll
            for (int j = 0; j < NR; ++j) tot[j] += __ldcg(partials + ((size_t)c * 32 + jj) * NR + j);
        if (!bs.done[jj] || !Fin::GATED) fin.finish(bs, jj, tot);
    }
    __syncthreads();
    if (threadIdx.x == 0) *bs.ticket = 0u;
}

// Row groups of the calling thread: (first row, stride) and its lane in the group.
#define FIIM_ROW_GROUPS(KP, row)                                                              \
    const int lane_ = threadIdx.x & 31, j_ = lane_ % (KP), grp_ = lane_ / (KP);               \
    const long gw_ = ((long)blockIdx.x * kThreads + threadIdx.x) >> 5;                        \
    const long nw_ = ((long)gridDim.x * kThreads) >> 5;                                       \
    for (long row = gw_ * (32 / (KP)) + grp_, base_ = gw_ * (32 / (KP));                      \
         base_ < sh.n; base_ += nw_ * (32 / (KP)), row = base_ + grp_)

// ---------------------------------------------------------------- epilogues
// emit(at, s, red) finishes entry `at` of the n x k output block from its row sum s;
// emit2(at, s0, s1, red0, red1) finishes the two consecutive entries at, at + 1 (at even)
// with the same arithmetic per entry, reading and writing both as one 16-byte pair (the
// sparse products with two or four right-hand sides per lane).
#define FIIM_BEPI(nr, reduces, gated)            \
    static constexpr int NR = nr;                \
    static constexpr bool REDUCES = reduces;     \
    static constexpr bool GATED = gated

__device__ __forceinline__ void st2(double *p, double a, double b) { *reinterpret_cast<double2 *>(p) = make_double2(a, b); }
__device__ __forceinline__ double2 ld2(const double *__restrict__ p) { return __ldg(reinterpret_cast<const double2 *>(p)); }

struct KEpiStore {
    FIIM_BEPI(1, false, true);
    double *y;
    __device__ void emit(size_t at, double s, double (&)[NR]) const { y[at] = s; }
    __device__ void emit2(size_t at, double s0, double s1, double (&)[NR], double (&)[NR]) const { st2(y + at, s0, s1); }
    __device__ void finish(BState &, int, const double *) const {}
};
struct KEpiScale {                 // y = d o (M x), d per row
    FIIM_BEPI(1, false, true);
    double *y;
    const double *__restrict__ d;
    int k;
    __device__ void emit(size_t at, double s, double (&)[NR]) const { y[at] = __dmul_rn(__ldg(d + at / k), s); }
    __device__ void emit2(size_t at, double s0, double s1, double (&)[NR], double (&)[NR]) const {
        const double di = __ldg(d + at / k);
        st2(y + at, __dmul_rn(di, s0), __dmul_rn(di, s1));
    }
    __device__ void finish(BState &, int, const double *) const {}
};
struct KEpiNorm {
    FIIM_BEPI(1, true, true);
    double *y;
    __device__ void emit(size_t at, double s, double (&r)[NR]) const { y[at] = s; r[0] += s * s; }
    __device__ void emit2(size_t at, double s0, double s1, double (&ra)[NR], double (&rb)[NR]) const {
        st2(y + at, s0, s1);
        ra[0] += s0 * s0;
        rb[0] += s1 * s1;
    }
    __device__ void finish(BState &bs, int j, const double *t) const { bs.pc2[j] = t[0]; }
};
struct KEpiAlpha {
    FIIM_BEPI(1, true, true);
    double *y;
    const double *__restrict__ r0;
    __device__ void emit(size_t at, double s, double (&r)[NR]) const {
        y[at] = s;
        r[0] += __ldg(r0 + at) * s;
    }
    __device__ void emit2(size_t at, double s0, double s1, double (&ra)[NR], double (&rb)[NR]) const {
        st2(y + at, s0, s1);
        const double2 q = ld2(r0 + at);
        ra[0] += q.x * s0;
        rb[0] += q.y * s1;
    }
    __device__ void finish(BState &bs, int j, const double *t) const { bt::BEpiAlpha{}.finish(bs, j, t); }
};
struct KEpiOmega {
    FIIM_BEPI(2, true, true);
    double *y;
    const double *__restrict__ sv;
    __device__ void emit(size_t at, double s, double (&r)[NR]) const {
        y[at] = s;
        r[0] += s * __ldg(sv + at);
        r[1] += s * s;
    }
    __device__ void emit2(size_t at, double s0, double s1, double (&ra)[NR], double (&rb)[NR]) const {
        st2(y + at, s0, s1);
        const double2 q = ld2(sv + at);
        ra[0] += s0 * q.x;
        ra[1] += s0 * s0;
        rb[0] += s1 * q.y;
        rb[1] += s1 * s1;
    }
    __device__ void finish(BState &bs, int j, const double *t) const { bs.omega[j] = t[0] / t[1]; }
};
struct KEpiInit {
    FIIM_BEPI(1, true, true);
    const double *__restrict__ b;
    double *p, *r0, *r;
    __device__ void emit(size_t at, double s, double (&red)[NR]) const {
        const double pi = __dadd_rn(b[at], __dmul_rn(-1.0, s));
        p[at] = pi;
        r0[at] = pi;
        r[at] = pi;
        red[0] += pi * pi;
    }
    __device__ void emit2(size_t at, double s0, double s1, double (&ra)[NR], double (&rb)[NR]) const {
        const double2 q = ld2(b + at);
        const double p0 = __dadd_rn(q.x, __dmul_rn(-1.0, s0)), p1 = __dadd_rn(q.y, __dmul_rn(-1.0, s1));
        st2(p + at, p0, p1);
        st2(r0 + at, p0, p1);
        st2(r + at, p0, p1);
        ra[0] += p0 * p0;
        rb[0] += p1 * p1;
    }
    __device__ void finish(BState &bs, int j, const double *t) const { bt::BFinInit{}.finish(bs, j, t); }
};
struct KEpiRestart : KEpiInit {
    __device__ void finish(BState &bs, int j, const double *t) const { bt::BFinRestart{}.finish(bs, j, t); }
};
struct KEpiResid {
    FIIM_BEPI(2, true, false);
    const double *__restrict__ b;
    __device__ void emit(size_t at, double s, double (&red)[NR]) const {
        const double bi = b[at], ri = bi - s;
        red[0] += ri * ri;
        red[1] += bi * bi;
    }
    __device__ void emit2(size_t at, double s0, double s1, double (&ra)[NR], double (&rb)[NR]) const {
        const double2 q = ld2(b + at);
        const double ri0 = q.x - s0, ri1 = q.y - s1;
        ra[0] += ri0 * ri0;
        ra[1] += q.x * q.x;
        rb[0] += ri1 * ri1;
        rb[1] += q.y * q.y;
    }
    __device__ void finish(BState &bs, int j, const double *t) const {
        bs.ts[j] = t[0];
        bs.tt[j] = t[1];
    }
};

__device__ __forceinline__ double wide(double v) { return v; }
__device__ __forceinline__ double wide(float v) { return (double)v; }

// ---------------------------------------------------------------- SpMM
// X's VW values of one gathered row for a lane, from a 16-byte aligned address when VW > 1
// (VW > 1 needs an even k and VW | k, so that row * k + l * VW is a multiple of VW).
template <int VW>
__device__ __forceinline__ void gather(const double *__restrict__ p, double (&x)[VW]) {
    if constexpr (VW == 1) {
        x[0] = __ldg(p);
    } else {
#pragma unroll
        for (int u = 0; u < VW; u += 2) {
            const double2 d = __ldg(reinterpret_cast<const double2 *>(p + u));
            x[u] = d.x;
            x[u + 1] = d.y;
        }
    }
}

template <int L, int VW, typename V, typename Epi>
static __global__ void __launch_bounds__(kThreads)
k_spmm(CsrView<V> M, Shape sh, const double *__restrict__ X, Epi epi, BState bs, double *__restrict__ partials) {
    if (Epi::GATED && bs.g->active <= 0) return;
    double red[VW][Epi::NR];
#pragma unroll
    for (int u = 0; u < VW; ++u)
#pragma unroll
        for (int q = 0; q < Epi::NR; ++q) red[u][q] = 0.0;
    FIIM_ROW_GROUPS(L, row) {
        const bool live = row < sh.n;
        const int j0 = j_ * VW;            // this lane's first right-hand side
        int beg = 0, len = 0;
        if (live) {
            beg = __ldg(M.rp + row);
            len = __ldg(M.rp + row + 1) - beg;
        }
        // every group of the warp walks the longest row of the warp (uniform shuffles), and
        // within a trip only as many entries as the longest remaining row part holds
        const int trips = __reduce_max_sync(0xffffffffu, (len + L - 1) / L);
        double s[VW];
#pragma unroll
        for (int u = 0; u < VW; ++u) s[u] = 0.0;
        for (int t = 0; t < trips; ++t) {
            const int q = t * L + j_;
            int c = 0;
            double a = 0.0;
            if (q < len) {
                c = ldi(M.ci + beg + q);
                a = wide(ldm(M.v + beg + q));
            }
            const int ne = (int)__reduce_max_sync(0xffffffffu, (unsigned)max(0, min(L, len - t * L)));
#pragma unroll 4
            for (int e = 0; e < ne; ++e) {
                const int ce = __shfl_sync(0xffffffffu, c, grp_ * L + e);
                const double ae = __shfl_sync(0xffffffffu, a, grp_ * L + e);
                if (t * L + e < len && j0 < sh.k) {
                    double xv[VW];
                    gather<VW>(X + (size_t)ce * sh.k + j0, xv);
#pragma unroll
                    for (int u = 0; u < VW; ++u) s[u] = __dadd_rn(s[u], __dmul_rn(ae, xv[u]));
                }
            }
        }
        if (live && j0 < sh.k) {
            const size_t at = (size_t)row * sh.k + j0;
            bool all = true;   // every right-hand side of this lane still running
            if constexpr (Epi::GATED)
#pragma unroll
                for (int u = 0; u < VW; ++u) all = all && !bs.done[j0 + u];
            if (VW > 1 && all) {
#pragma unroll
                for (int u = 0; u < VW; u += 2) epi.emit2(at + u, s[u], s[u + 1], red[u], red[u + 1]);
            } else {
#pragma unroll
                for (int u = 0; u < VW; ++u)
                    if (!(Epi::GATED && bs.done[j0 + u])) epi.emit(at + u, s[u], red[u]);
            }
        }
    }
    if constexpr (Epi::REDUCES) rhs_reduce<L, VW, Epi::NR>(red, sh.k, partials, bs, epi);
}

// ---------------------------------------------------------------- updates (n x k)
struct KFinS {
    static constexpr bool GATED = true;
    __device__ void finish(BState &bs, int j, const double *t) const { bt::BFinS{}.finish(bs, j, t); }
};
struct KFinControl {
    static constexpr bool GATED = true;
    __device__ void finish(BState &bs, int j, const double *t) const { bt::BFinControl{}.finish(bs, j, t); }
};

template <int KP>
static __global__ void __launch_bounds__(kThreads)
k_kupdate_s(Shape sh, const double *__restrict__ r, const double *__restrict__ v, const double *__restrict__ x,
            double *__restrict__ s, BState bs, double *__restrict__ partials) {
    if (bs.g->active <= 0) return;
    double red[1][2] = {{0.0, 0.0}};
    FIIM_ROW_GROUPS(KP, row) {
        if (row >= sh.n || j_ >= sh.k || bs.done[j_]) continue;
        const size_t at = (size_t)row * sh.k + j_;
        const double ri = r[at], xi = x[at];
        s[at] = __dadd_rn(ri, __dmul_rn(-bs.alpha[j_], v[at]));
        red[0][0] += ri * ri;
        red[0][1] += xi * xi;
    }
    rhs_reduce<KP, 1, 2>(red, sh.k, partials, bs, KFinS{});
}

template <int KP>
static __global__ void __launch_bounds__(kThreads)
k_kupdate_xr(Shape sh, const double *__restrict__ pc, const double *__restrict__ sc, const double *__restrict__ s,
             const double *__restrict__ t, const double *__restrict__ r0, double *__restrict__ x,
             double *__restrict__ r, BState bs, double *__restrict__ partials) {
    if (bs.g->active <= 0) return;
    double red[1][1] = {{0.0}};
    FIIM_ROW_GROUPS(KP, row) {
        if (row >= sh.n || j_ >= sh.k || bs.done[j_]) continue;
        const size_t at = (size_t)row * sh.k + j_;
        const double a = bs.alpha[j_], om = bs.omega[j_];
        double xi = x[at];
        xi = __dadd_rn(xi, __dmul_rn(a, pc[at]));
        xi = __dadd_rn(xi, __dmul_rn(om, sc[at]));
        x[at] = xi;
        const double ri = __dadd_rn(s[at], __dmul_rn(-om, t[at]));
        r[at] = ri;
        red[0][0] += r0[at] * ri;
    }
    rhs_reduce<KP, 1, 1>(red, sh.k, partials, bs, KFinControl{});
}

template <int KP>
static __global__ void __launch_bounds__(kThreads)
k_kupdate_p(Shape sh, const double *__restrict__ r, const double *__restrict__ v, double *__restrict__ p, BState bs,
            cudaGraphConditionalHandle h, int cond) {
    if (cond && blockIdx.x == 0 && threadIdx.x == 0) {
        const int loops = ++bs.g->loops;
        if (bs.g->active > 0 && loops > bs.g->nmax + 2) bs.g->active = -1;
        cudaGraphSetConditional(h, bs.g->active > 0 ? 1u : 0u);
    }
    if (bs.g->active <= 0) return;
    FIIM_ROW_GROUPS(KP, row) {
        if (row >= sh.n || j_ >= sh.k || bs.done[j_]) continue;
        const size_t at = (size_t)row * sh.k + j_;
        const double b = bs.beta[j_], c = __dmul_rn(-bs.beta[j_], bs.omega[j_]);
        const double pi = __dadd_rn(__dmul_rn(c, v[at]), __dmul_rn(b, p[at]));
        p[at] = __dadd_rn(pi, r[at]);
    }
}

}  // namespace bk
}  // namespace fiim
