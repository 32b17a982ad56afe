// The whole FP64 solve in one cooperative launch, for small systems (sm_100a; FIIM_PERSIST=1).
//
// At small n every kernel of the iteration body finishes in a few microseconds, and the
// solve is bound by launch and reduction latency (≈ 4 µs per launch at n = 16,384). Here one
// cooperative grid runs the start step, the iteration loop and the true residual as phases
// separated by a grid barrier, so a launch becomes a barrier. On B200 the barrier and the
// exchange of partial sums cost as much as a launch with programmatic dependent launch in a
// CUDA graph: Poisson 128^2 runs 41.7 µs per iteration this way against 34.7 µs for the WHILE
// graph, so the graph stays the default.
//
// The arithmetic is that of the launched kernels: each SpMV row is summed left to right in
// storage order with rounded products (the CSR-stream row blocks of the solver), the
// epilogues are the same objects, and the vector updates round their products and sums
// exactly as k_update_s / k_update_xr / k_update_p do. The dot products are reduced over the
// CTAs of this grid (a fixed tree, deterministic), so they round differently from the launched
// kernels' trees, as those differ between launch shapes.
//
// Reductions: each CTA writes its partial sums, alternating between two buffers; after the
// barrier every CTA adds all CTAs' partials in CTA order into its own shared copy of the solve
// scalars and applies the scalar step there, so every CTA holds the same scalars and takes the
// same branches, and no second barrier is needed. CTA 0 stores the scalars for the host.
//
// The barrier's wait is bounded: past the limit it sets *fault and the CTA leaves the solve;
// every other CTA then runs out at the same or the next barrier. The host turns the flag into
// FIIM_ETIMEOUT.
#pragma once

#include "fiim_kernels.cuh"

namespace fiim {

struct PView {   // one CSR matrix with its row blocks and optional 16-bit column stream
    const int *rp, *ci;
    const double *v;
    const int *rb, *eb;
    int nblk;
    const short *cd;
    const int *cb;
    int narrow;
};

struct PersistArgs {
    PView A, G, H;
    int n;
    double *x, *b, *r, *r0, *p, *v, *s, *t, *pc, *sc, *tm;
    const double *IDv;
    DState *st;                 // in: the solve's parameters; out: the final scalars
    double *partials;           // 2 buffers of gridDim.x * 4
    unsigned *bar;              // [0] arrivals, [1] generation
    int *fault;
    int wait_limit;             // barrier polls before giving up
};

constexpr int kPTile = 2048;

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Bounded grid barrier (one arrival counter and a generation word). The generation is read
// before arriving, so the last arrival cannot advance it unseen.
__device__ __forceinline__ bool pgrid_sync(const PersistArgs &a) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        const unsigned g = ld_acquire(a.bar + 1);
        __threadfence();
        if (atomicAdd(a.bar, 1u) == gridDim.x - 1) {
            atomicExch(a.bar, 0u);
            __threadfence();
            atomicAdd(a.bar + 1, 1u);
        } else {
            int i = 0;
            while (ld_acquire(a.bar + 1) == g) {
                if (++i > a.wait_limit) {
                    atomicExch(a.fault, 1);
                    ok = 0;
                    break;
                }
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok;
}

// One SpMV over the matrix's row blocks (CTA per block, grid-stride): products rounded into
// shared memory, each row summed left to right by its thread, the epilogue emitting. Vectors
// change between the phases of this one kernel, so they are read through L2 (ld.global.cg),
// never through the non-coherent read-only path the launched kernels use; the epilogue's
// per-row operand is loaded here for the same reason.
template <typename Epi>
__device__ __forceinline__ void pemit(const Epi &epi, long i, double s, double (&red)[Epi::NR]) {
    if constexpr (HasPre<Epi>::value) epi.emit_pre(i, s, __ldcg(epi.pre_ptr() + i), red);
    else epi.emit(i, s, red);
}

template <bool NARROW, typename Epi>
__device__ __forceinline__ void pspmv(const PView &M, const double *__restrict__ x, const Epi &epi, double (&red)[Epi::NR],
                      double *prod) {
    const int tid = (int)threadIdx.x;
    for (int blk = blockIdx.x; blk < M.nblk; blk += gridDim.x) {
        const int r0 = M.rb[blk], r1 = M.rb[blk + 1], e0 = M.eb[blk], e1 = M.eb[blk + 1];
        const int cbs = NARROW ? M.cb[blk] : 0;
        auto col = [&](int e) { return NARROW ? cbs + (int)M.cd[e] : M.ci[e]; };
        if (e1 - e0 < kPTile) {
            for (int e = e0 + tid; e < e1; e += kThreads) prod[e - e0] = __dmul_rn(M.v[e], __ldcg(x + col(e)));
            __syncthreads();
            const int r = r0 + tid;
            if (r < r1) {
                double sum = 0.0;
                for (int k = M.rp[r] - e0; k < M.rp[r + 1] - e0; ++k) sum = __dadd_rn(sum, prod[k]);
                pemit(epi, r, sum, red);
            }
            __syncthreads();
        } else {
            double sum = 0.0;
            for (int c0 = e0; c0 < e1; c0 += kPTile) {
                const int c1 = min(c0 + kPTile, e1);
                for (int e = c0 + tid; e < c1; e += kThreads) prod[e - c0] = __dmul_rn(M.v[e], __ldcg(x + col(e)));
                __syncthreads();
                if (tid == 0)
                    for (int k = 0; k < c1 - c0; ++k) sum = __dadd_rn(sum, prod[k]);
                __syncthreads();
            }
            if (tid == 0) pemit(epi, r0, sum, red);
        }
    }
}

template <typename Epi>
__device__ __forceinline__ void pspmv_any(const PView &M, const double *x, const Epi &epi, double (&red)[Epi::NR],
                                          double *prod) {
    if (M.narrow) pspmv<true>(M, x, epi, red, prod);
    else pspmv<false>(M, x, epi, red, prod);
}

// This CTA's partial sums (fixed tree) into buffer `buf`; after the barrier, every CTA's sums
// in CTA order, then fin.finish on the CTA's shared scalars. False if the barrier gave up.
template <int NR, class Fin>
__device__ __forceinline__ bool preduce(const PersistArgs &a, double (&v)[NR], int buf, DState *sst, const Fin &fin) {
    __shared__ double sm[kWarps][4];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < NR; ++j) v[j] = warp_sum(v[j]);
    if (lane == 0)
#pragma unroll
        for (int j = 0; j < NR; ++j) sm[w][j] = v[j];
    __syncthreads();
    double *P = a.partials + (size_t)buf * gridDim.x * 4;
    if (threadIdx.x == 0)
#pragma unroll
        for (int j = 0; j < NR; ++j) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < kWarps; ++k) s += sm[k][j];
            P[(size_t)blockIdx.x * 4 + j] = s;
        }
    if (!pgrid_sync(a)) return false;
    if (w == 0) {
        double acc[NR];
#pragma unroll
        for (int j = 0; j < NR; ++j) acc[j] = 0.0;
        for (int k = lane; k < (int)gridDim.x; k += 32)
#pragma unroll
            for (int j = 0; j < NR; ++j) acc[j] += __ldcg(P + (size_t)k * 4 + j);
#pragma unroll
        for (int j = 0; j < NR; ++j) acc[j] = warp_sum(acc[j]);
        if (lane == 0) fin.finish(sst, acc);
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < NR; ++j) v[j] = 0.0;
    return true;
}

static __global__ void __launch_bounds__(kThreads) k_solve_persistent(PersistArgs a) {
    __shared__ double prod[kPTile];
    __shared__ DState sst;
    const int n = a.n;
    if (threadIdx.x == 0) sst = *a.st;
    __syncthreads();
    int buf = 0;
    auto rows = [&](auto f) {
        for (long i = (long)blockIdx.x * kThreads + threadIdx.x; i < n; i += (long)gridDim.x * kThreads) f(i);
    };
    // Start: r = b - A x, r0 = r, p = r, ro = ||r0|| (AFIIM/src/bicgstab.cpp:151-165).
    {
        double red[1] = {0.0};
        pspmv_any(a.A, a.x, EpiInit{a.b, a.p, a.r0, a.r}, red, prod);
        if (!preduce<1>(a, red, buf ^= 1, &sst, FinInit{})) return;   // its barrier completes p, r0, r
    }
    for (;;) {
        if (sst.done) break;
        // tm = D^-1 o (H p); pc = G tm, ||pc||^2; v = A pc, alpha (:172-181)
        {
            double red[1] = {0.0};
            pspmv_any(a.H, a.p, EpiScale{a.tm, a.IDv}, red, prod);
            if (!pgrid_sync(a)) return;
            pspmv_any(a.G, a.tm, EpiNorm{a.pc}, red, prod);
            if (!preduce<1>(a, red, buf ^= 1, &sst, EpiNorm{a.pc})) return;
            pspmv_any(a.A, a.pc, EpiAlpha{a.v, a.r0}, red, prod);
            if (!preduce<1>(a, red, buf ^= 1, &sst, EpiAlpha{a.v, a.r0})) return;
        }
        if (sst.done) break;   // non-finite alpha (ACIFIM)
        // s = r - alpha v, ||r||^2, ||x||^2 (:184-185, :201, :216)
        {
            double red[2] = {0.0, 0.0};
            const double na = -sst.alpha;
            rows([&](long i) {
                const double ri = __ldcg(a.r + i), xi = __ldcg(a.x + i);
                a.s[i] = __dadd_rn(ri, __dmul_rn(na, __ldcg(a.v + i)));
                red[0] += ri * ri;
                red[1] += xi * xi;
            });
            if (!preduce<2>(a, red, buf ^= 1, &sst, FinS{})) return;
        }
        // tm = D^-1 o (H s); sc = G tm; t = A sc, omega (:189-198)
        {
            double red[2] = {0.0, 0.0};
            double red1[1] = {0.0};
            pspmv_any(a.H, a.s, EpiScale{a.tm, a.IDv}, red1, prod);
            if (!pgrid_sync(a)) return;
            pspmv_any(a.G, a.tm, EpiStore{a.sc}, red1, prod);
            if (!pgrid_sync(a)) return;
            pspmv_any(a.A, a.sc, EpiOmega{a.t, a.s}, red, prod);
            if (!preduce<2>(a, red, buf ^= 1, &sst, EpiOmega{a.t, a.s})) return;
        }
        // x += alpha pc + omega sc; r = s - omega t; r0 . r; tests and beta (:207-274)
        {
            double red[1] = {0.0};
            const double al = sst.alpha, om = sst.omega, nom = -sst.omega;
            rows([&](long i) {
                double xi = __ldcg(a.x + i);
                xi = __dadd_rn(xi, __dmul_rn(al, __ldcg(a.pc + i)));
                xi = __dadd_rn(xi, __dmul_rn(om, __ldcg(a.sc + i)));
                a.x[i] = xi;
                const double ri = __dadd_rn(__ldcg(a.s + i), __dmul_rn(nom, __ldcg(a.t + i)));
                a.r[i] = ri;
                red[0] += __ldcg(a.r0 + i) * ri;
            });
            if (!preduce<1>(a, red, buf ^= 1, &sst, FinControl{})) return;
        }
        if (sst.done) break;
        // p = (-beta omega) v + beta p; p = p + r (:270-271)
        {
            const double bb = sst.beta, c = __dmul_rn(-sst.beta, sst.omega);
            rows([&](long i) {
                const double pi = __dadd_rn(__dmul_rn(c, __ldcg(a.v + i)), __dmul_rn(bb, __ldcg(a.p + i)));
                a.p[i] = __dadd_rn(pi, __ldcg(a.r + i));
            });
            if (!pgrid_sync(a)) return;
        }
    }
    // FP64 true residual ||b - A x|| / ||b||, then the scalars for the host.
    if (!pgrid_sync(a)) return;   // x complete
    {
        double red[2] = {0.0, 0.0};
        pspmv_any(a.A, a.x, EpiResid{a.b, nullptr}, red, prod);
        if (!preduce<2>(a, red, buf ^= 1, &sst, EpiResid{a.b, nullptr})) return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *a.st = sst;
}

}  // namespace fiim
