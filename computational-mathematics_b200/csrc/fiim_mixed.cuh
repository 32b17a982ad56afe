// Device kernels of the mixed-precision solve: FP64 iterative refinement around an FP32
// inner BiCGSTAB with the same control flow as the reference's loop
// (AFIIM/src/bicgstab.cpp:168-275), on FP32 vectors and FP32 (or BF16) matrix values.
//
// Inner iteration = the nine launches of the FP64 path, on 4-byte vectors:
//   tm = D^{-1} o (H p); pc = G tm (+||pc||^2); v = A32 pc, alpha; s = r - alpha v (+||r||^2,
//   ||e||^2); tm = D^{-1} o (H s); sc = G tm; t = A32 sc, omega; e += alpha pc + omega sc,
//   r = s - omega t, m1 = r0.r, tests, beta; p = r + beta (p - omega v).
// Matrix products accumulate in FP32 (rows summed in storage order from shared memory);
// every dot product and norm accumulates FP32 products in FP64, and the recurrence scalars
// (alpha, omega, beta, rho) are FP64 in DState.
//
// Outer step (FP64): r64 = b - A x with the FP64 A (the FP64 kernel's EpiResid), the inner
// solve runs on r64 / ||r64|| from e = 0, then x += ||r64|| e.
#pragma once

#include "fiim_kernels.cuh"

namespace fiim {
namespace mx {

// ---------------------------------------------------------------- FP32 epilogues
struct EpiStoreF {
    FIIM_EPI(1, false, true);
    float *y;
    __device__ void emit(long i, float s, double (&)[NR]) const { y[i] = s; }
    __device__ void finish(DState *, const double *) const {}
};
struct EpiScaleF {                 // y = d o (M x)
    FIIM_EPI(1, false, true);
    float *y;
    const float *__restrict__ d;
    __device__ const float *pre_ptr() const { return d; }
    __device__ float pre(long i) const { return __ldg(d + i); }
    __device__ void emit_pre(long i, float s, float di, double (&)[NR]) const { y[i] = di * s; }
    __device__ void emit(long i, float s, double (&r)[NR]) const { emit_pre(i, s, pre(i), r); }
    __device__ void finish(DState *, const double *) const {}
};
struct EpiNormF {                  // y = M x, ||y||^2 -> st->pc2
    FIIM_EPI(1, true, true);
    float *y;
    __device__ void emit(long i, float s, double (&r)[NR]) const {
        y[i] = s;
        r[0] += (double)s * (double)s;
    }
    __device__ void finish(DState *st, const double *t) const { st->pc2 = t[0]; }
};
struct EpiAlphaF {                 // v = A pc, alpha = m1 / (r0 . v)
    FIIM_EPI(1, true, true);
    float *y;
    const float *__restrict__ r0;
    __device__ const float *pre_ptr() const { return r0; }
    __device__ float pre(long i) const { return __ldg(r0 + i); }
    __device__ void emit_pre(long i, float s, float r0i, double (&r)[NR]) const {
        y[i] = s;
        r[0] += (double)r0i * (double)s;
    }
    __device__ void emit(long i, float s, double (&r)[NR]) const { emit_pre(i, s, pre(i), r); }
    __device__ void finish(DState *st, const double *t) const { EpiAlpha{nullptr, nullptr}.finish(st, t); }
};
struct EpiOmegaF {                 // t = A sc, omega = (t . s) / (t . t)
    FIIM_EPI(2, true, true);
    float *y;
    const float *__restrict__ sv;
    __device__ const float *pre_ptr() const { return sv; }
    __device__ float pre(long i) const { return __ldg(sv + i); }
    __device__ void emit_pre(long i, float s, float si, double (&r)[NR]) const {
        y[i] = s;
        r[0] += (double)s * (double)si;
        r[1] += (double)s * (double)s;
    }
    __device__ void emit(long i, float s, double (&r)[NR]) const { emit_pre(i, s, pre(i), r); }
    __device__ void finish(DState *st, const double *t) const { EpiOmega{nullptr, nullptr}.finish(st, t); }
};

__device__ __forceinline__ float ldv(const float *p) { return __ldcs(p); }
__device__ __forceinline__ float ldv(const __nv_bfloat16 *p) { return ldm(p); }

// CSR-stream SpMV on FP32 / BF16 values and an FP32 vector, with the FP64 kernel's row
// blocks (at most TILE - 1 entries, bounds rb / eb), column streams (32-bit or NARROW) and
// structure: entries read in aligned
// pairs, the next block's bounds, row offsets, entry streams and epilogue operands loaded
// into registers before the barrier, products staged in shared memory, each row summed in
// storage order.
template <int TILE, typename V, typename Epi, bool NARROW = false>
static __global__ void __launch_bounds__(kThreads)
k_spmv_rows_f(CsrView<V> M, const int *__restrict__ rb, const int *__restrict__ eb, int nblk,
              const float *__restrict__ x, Epi epi, DState *st, double *__restrict__ partials,
              NarrowCols nc = NarrowCols{}) {
    pdl_enter();
    if (Epi::GATED && st != nullptr && st->done) return;
    __shared__ float prod[TILE];
    constexpr int PER = TILE / kThreads;
    const int tid = (int)threadIdx.x;
    double red[Epi::NR];
#pragma unroll
    for (int j = 0; j < Epi::NR; ++j) red[j] = 0.0;
    int r0 = 0, r1 = 0, e0 = 0, e1 = 0, rbeg = 0, rend = 0, cbase = 0;
    float opnd = 0.f;
    using VP = ValPair<V>;
    ColRegs<NARROW, PER> c;
    typename VP::T a[PER / 2];
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
        const float copnd = opnd;
        if (ce1 - ce0 < TILE) {
            const int a0 = ce0 & ~1;
#pragma unroll
            for (int u = 0; u < PER; ++u) {
                const int e = a0 + 2 * (tid + (u >> 1) * kThreads) + (u & 1);
                if (e >= ce0 && e < ce1) prod[e - ce0] = VP::get(a[u >> 1], u & 1) * ldx(x + c.get(u, cbs));
            }
            if (nxt < nblk) fetch(nxt);
            __syncthreads();
            if (cr0 + tid < cr1) {
                float s = 0.f;
                for (int k = cb; k < ce; ++k) s += prod[k];
                if constexpr (HasPre<Epi>::value) epi.emit_pre(cr0 + tid, s, copnd, red);
                else epi.emit(cr0 + tid, s, red);
            }
            __syncthreads();
        } else {
            float s = 0.f;
            for (int c0 = ce0; c0 < ce1; c0 += TILE) {
                const int c1 = min(c0 + TILE, ce1);
                for (int e = c0 + tid; e < c1; e += kThreads) {
                    const int j = NARROW ? cbs + (int)__ldcs(nc.d + e) : ldi(M.ci + e);
                    prod[e - c0] = ldv(M.v + e) * ldx(x + j);
                }
                __syncthreads();
                if (tid == 0)
                    for (int k = 0; k < c1 - c0; ++k) s += prod[k];
                __syncthreads();
            }
            if (tid == 0) epi.emit(cr0, s, red);
            if (nxt < nblk) fetch(nxt);
        }
    }
    pdl_release();
    if constexpr (Epi::REDUCES) grid_reduce<Epi::NR>(red, partials, st, epi);
}

// ---------------------------------------------------------------- inner start / updates
// Grid-stride over the rows four at a time (one 16-byte load of each FP32 vector: the arena
// keeps them 256-byte aligned), then the last n % 4 rows one at a time. f4(q) handles rows
// 4q .. 4q + 3, f1(i) row i. The FP32 updates move few bytes a launch; one float a thread a
// step left them at 3-4.5 TB/s under ncu.
__device__ __forceinline__ float4 ld4(const float *p, long q) { return reinterpret_cast<const float4 *>(p)[q]; }
__device__ __forceinline__ void st4(float *p, long q, float4 v) { reinterpret_cast<float4 *>(p)[q] = v; }
template <class F4, class F1>
__device__ __forceinline__ void rows4(long n, F4 f4, F1 f1) {
    const long n4 = n >> 2, stride = (long)gridDim.x * kThreads, t = (long)blockIdx.x * kThreads + threadIdx.x;
    for (long q = t; q < n4; q += stride) f4(q);
    for (long i = 4 * n4 + t; i < n; i += stride) f1(i);
}

// Inner start from e = 0: r = r0 = p = r64 / ||r64|| in FP32 (||r64||^2 is sto->ts from
// the residual kernel); ||r0||^2 accumulated in FP64 -> ro, m1, rc (FinInit).
static __global__ void __launch_bounds__(kThreads)
k_inner_init(long n, const double *__restrict__ r64, const DState *sto, float *__restrict__ r,
             float *__restrict__ r0, float *__restrict__ p, float *__restrict__ e, DState *st,
             double *__restrict__ partials) {
    pdl_enter();
    const double inv = 1.0 / sqrt(sto->ts);
    double red[1] = {0.0};
    FIIM_FOR_ROWS(i, n) {
        const float ri = (float)(r64[i] * inv);
        r[i] = ri;
        r0[i] = ri;
        p[i] = ri;
        e[i] = 0.f;
        red[0] += (double)ri * (double)ri;
    }
    pdl_release();
    grid_reduce<1>(red, partials, st, FinInit{});
}

static __global__ void __launch_bounds__(kThreads)
k_update_s_f(long n, const float *__restrict__ r, const float *__restrict__ v,
             const float *__restrict__ e, float *__restrict__ s, DState *st,
             double *__restrict__ partials) {
    pdl_enter();
    if (st->done) return;
    const float na = (float)(-st->alpha);
    double red[2] = {0.0, 0.0};
    auto row = [&](float ri, float vi, float ei) {
        red[0] += (double)ri * (double)ri;
        red[1] += (double)ei * (double)ei;
        return fmaf(na, vi, ri);
    };
    rows4(
        n,
        [&](long q) {
            const float4 r4 = ld4(r, q), v4 = ld4(v, q), e4 = ld4(e, q);
            st4(s, q, make_float4(row(r4.x, v4.x, e4.x), row(r4.y, v4.y, e4.y), row(r4.z, v4.z, e4.z),
                                  row(r4.w, v4.w, e4.w)));
        },
        [&](long i) { s[i] = row(r[i], v[i], e[i]); });
    pdl_release();
    grid_reduce<2>(red, partials, st, FinS{});
}

template <class Fin = FinControl>
static __global__ void __launch_bounds__(kThreads)
k_update_xr_f(long n, const float *__restrict__ pc, const float *__restrict__ sc,
              const float *__restrict__ s, const float *__restrict__ t,
              const float *__restrict__ r0, float *__restrict__ e, float *__restrict__ r,
              DState *st, double *__restrict__ partials, Fin fin = Fin{}) {
    pdl_enter();
    if (st->done) return;
    const float a = (float)st->alpha, om = (float)st->omega;
    double red[1] = {0.0};
    auto res = [&](float si, float ti, float r0i) {   // r = s - omega t; r0 . r
        const float ri = fmaf(-om, ti, si);
        red[0] += (double)r0i * (double)ri;
        return ri;
    };
    auto cor = [&](float ei, float pci, float sci) { return fmaf(om, sci, fmaf(a, pci, ei)); };   // e update
    rows4(
        n,
        [&](long q) {
            const float4 e4 = ld4(e, q), pc4 = ld4(pc, q), sc4 = ld4(sc, q), s4 = ld4(s, q), t4 = ld4(t, q),
                         q4 = ld4(r0, q);
            st4(e, q, make_float4(cor(e4.x, pc4.x, sc4.x), cor(e4.y, pc4.y, sc4.y), cor(e4.z, pc4.z, sc4.z),
                                  cor(e4.w, pc4.w, sc4.w)));
            st4(r, q, make_float4(res(s4.x, t4.x, q4.x), res(s4.y, t4.y, q4.y), res(s4.z, t4.z, q4.z),
                                  res(s4.w, t4.w, q4.w)));
        },
        [&](long i) {
            e[i] = cor(e[i], pc[i], sc[i]);
            r[i] = res(s[i], t[i], r0[i]);
        });
    pdl_release();
    grid_reduce<1>(red, partials, st, fin);
}

static __global__ void __launch_bounds__(kThreads)
k_update_p_f(long n, const float *__restrict__ r, const float *__restrict__ v,
             float *__restrict__ p, DState *st, cudaGraphConditionalHandle h, int cond) {
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
    const float b = (float)st->beta, c = (float)(-st->beta * st->omega);
    auto dir = [&](float ri, float vi, float pi) { return fmaf(c, vi, fmaf(b, pi, ri)); };
    rows4(
        n,
        [&](long q) {
            const float4 r4 = ld4(r, q), v4 = ld4(v, q), p4 = ld4(p, q);
            st4(p, q, make_float4(dir(r4.x, v4.x, p4.x), dir(r4.y, v4.y, p4.y), dir(r4.z, v4.z, p4.z),
                                  dir(r4.w, v4.w, p4.w)));
        },
        [&](long i) { p[i] = dir(r[i], v[i], p[i]); });
}

// ---------------------------------------------------------------- reliable updates
// Residual replacement (Sleijpen and van der Vorst, "Reliable updated residuals in hybrid
// Bi-CG methods", Computing 56 (1996); in the mixed-precision form of Clark et al., "Solving
// lattice QCD systems of equations using mixed precision solvers on GPUs", Comput. Phys.
// Commun. 181 (2010)): ONE FP32 BiCGSTAB on (b - A x0) / sigma, sigma = ||b - A x0||, whose
// recurrence residual r is replaced by the FP64 true residual whenever ||r|| has fallen
// below delta times its largest value since the last replacement, and whenever the
// recurrence meets the target. A replacement first moves the correction into the FP64
// iterate (x += sigma e, e = 0), then computes b - A x with the FP64 A and sets
//   r <- (b - A x) / sigma,   p <- p + (r_new - r_old),   m1 <- r0 . r_new,
// so p is the direction the iteration would have formed from the new r, and the search
// directions are kept (a refinement step starts the Krylov space again). The solve stops
// only on the FP64 test ||b - A x|| <= tol ||b||, checked at a replacement.
struct RState {
    double sigma;      // scale of the FP32 vectors: ||b - A x0||
    double inv_sigma;  // 1 / sigma
    double goal;       // the FP64 target on ||b - A x||: tol ||b||
    double delta;      // replace when ||r|| < delta * rmax
    double rmax;       // largest recurrence ||r|| (scaled) since the last replacement
    double true_r;     // ||b - A x|| at the last replacement
    int update;        // replace at the end of this body
    int verify;        // the recurrence met the target: the replacement decides the stop
    int replacements, verifies, max_verify;
};

// FinControl's tests (AFIIM/src/bicgstab.cpp:201-277) with the recurrence's convergence
// test turned into a request for a replacement (the FP64 residual decides the stop), and
// the replacement trigger: ||r|| below delta times its running maximum.
struct FinControlR {
    RState *rs;
    __device__ void finish(DState *st, const double *t) const {
        const double a = st->alpha, om = st->omega;
        if (fabs(a) * sqrt(st->pc2) < st->eps * sqrt(st->x2)) st->stag++;
        else st->stag = 0;
        const double prc = st->rc;
        st->rc = sqrt(st->r2);
        if (prc < st->rc) st->msteps++;
        else st->msteps = 0;
        if (st->msteps >= st->maxmsteps) { st->info = 1; st->done = 1; return; }
        if (st->stag >= 3) { st->info = 2; st->done = 1; return; }
        st->m2 = st->m1;
        st->m1 = t[0];
        st->beta = st->m1 * a / (om * st->m2);
        st->iter++;
        rs->rmax = fmax(rs->rmax, st->rc);
        if (st->rc < st->tol * st->ro) {
            rs->update = 1;
            rs->verify = 1;
        } else if (st->rc < rs->delta * rs->rmax) {
            rs->update = 1;
        }
        if (st->iter >= st->nmax) { st->info = 3; st->done = 1; }
    }
};

// p = r + beta (p - omega v), the last kernel of the body. cond bit 1: block 0 sets the IF
// node's condition (a replacement follows); bit 0 (the device-driven loop): it also counts
// the body, trips the guard (info -5) past nmax + 2 bodies and sets the WHILE node's
// condition. cond = 0 outside a graph: no condition is set.
static __global__ void __launch_bounds__(kThreads)
k_update_p_r(long n, const float *__restrict__ r, const float *__restrict__ v, float *__restrict__ p,
             DState *st, const RState *rs, cudaGraphConditionalHandle hw, cudaGraphConditionalHandle hif,
             int cond) {
    pdl_enter();
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (cond & 1) {   // inside the WHILE node's body
            const int loops = ++st->loops;
            if (!st->done && loops > st->nmax + 2) {
                st->info = -5;
                st->done = 1;
            }
            cudaGraphSetConditional(hw, st->done ? 0u : 1u);
        }
        if (cond & 2) cudaGraphSetConditional(hif, (!st->done && rs->update) ? 1u : 0u);   // the IF node follows
    }
    if (st->done) return;
    const float b = (float)st->beta, c = (float)(-st->beta * st->omega);
    auto dir = [&](float ri, float vi, float pi) { return fmaf(c, vi, fmaf(b, pi, ri)); };
    rows4(
        n,
        [&](long q) {
            const float4 r4 = ld4(r, q), v4 = ld4(v, q), p4 = ld4(p, q);
            st4(p, q, make_float4(dir(r4.x, v4.x, p4.x), dir(r4.y, v4.y, p4.y), dir(r4.z, v4.z, p4.z),
                                  dir(r4.w, v4.w, p4.w)));
        },
        [&](long i) { p[i] = dir(r[i], v[i], p[i]); });
}

// Replacement, first half: x += sigma e (FP64), e = 0.
static __global__ void __launch_bounds__(kThreads)
k_replace_x(long n, float *__restrict__ e, double *__restrict__ x, const RState *rs) {
    pdl_enter();
    const double scale = rs->sigma;
    FIIM_FOR_ROWS(i, n) {
        x[i] += scale * (double)e[i];
        e[i] = 0.f;
    }
}

// Replacement, second half: the epilogue of the FP64 product A x. Per row, the true
// residual b - A x (FP64), the new scaled FP32 residual, p moved by the change in r; sums
// ||b - A x||^2 and r0 . r_new. The finish sets m1, restarts the running maximum, and at a
// verification ends the solve when the FP64 target is met (or after max_verify attempts).
struct EpiReplace {
    FIIM_EPI(2, true, false);
    const double *__restrict__ b;
    float *r;
    float *p;
    const float *__restrict__ r0;
    RState *rs;
    __device__ void emit(long i, double s, double (&red)[NR]) const {
        const double rt = b[i] - s;
        const float rn = (float)(rt * rs->inv_sigma);
        p[i] += rn - r[i];
        r[i] = rn;
        red[0] += rt * rt;
        red[1] += (double)r0[i] * (double)rn;
    }
    __device__ void finish(DState *st, const double *t) const {
        rs->true_r = sqrt(t[0]);
        st->m1 = t[1];
        rs->rmax = rs->true_r * rs->inv_sigma;
        rs->update = 0;
        rs->replacements++;
        if (rs->verify) {
            rs->verify = 0;
            rs->verifies++;
            if (rs->true_r <= rs->goal) {
                st->info = 0;
                st->done = 1;
            } else if (rs->verifies >= rs->max_verify) {
                st->info = 3;
                st->done = 1;
            }
        }
    }
};

// x += ||r64|| e (FP64): the refinement step.
static __global__ void __launch_bounds__(kThreads)
k_promote(long n, const float *__restrict__ e, double *__restrict__ x, const DState *sto) {
    pdl_enter();
    const double scale = sqrt(sto->ts);
    FIIM_FOR_ROWS(i, n) { x[i] += scale * (double)e[i]; }
}

// Matrix values to the inner precision (round to nearest).
static __global__ void __launch_bounds__(kThreads)
k_to_f32(long n, const double *__restrict__ in, float *__restrict__ out) {
    FIIM_FOR_ROWS(i, n) { out[i] = __double2float_rn(in[i]); }
}
static __global__ void __launch_bounds__(kThreads)
k_to_bf16(long n, const double *__restrict__ in, __nv_bfloat16 *__restrict__ out) {
    FIIM_FOR_ROWS(i, n) { out[i] = __double2bfloat16(in[i]); }
}

}  // namespace mx
}  // namespace fiim
