// The whole FP64 solve of a small system in one thread-block cluster (sm_100a; FIIM_PERSIST=cluster).
//
// A small system (n <= kClusterCtas * kClusterMaxRows) is bound by launch and reduction
// latency, not bandwidth: at n = 16,384 each of the nine launches of an iteration costs about
// 4 us. Here one cluster of kClusterCtas CTAs runs the start step, the iteration loop and the
// true residual. CTA c owns the rows [c R, (c + 1) R) and keeps its part of every solve vector
// in its shared memory. The cluster's shared memory is addressable by every CTA of the
// cluster, so a product gathers the entries of other CTAs' rows from their shared memory
// directly; the matrices are streamed from global memory (L2). Phases are separated by the
// hardware cluster barrier in place of a kernel launch or a software grid barrier.
//
// The arithmetic is that of the launched kernels: one thread per row sums the row's rounded
// products left to right in storage order (every product and sum rounded on its own), the
// epilogues and vector updates round exactly as theirs do, and the scalar steps are the same
// objects (FinInit, FinS, FinControl and the epilogues' finish). The dot products are reduced
// in a fixed tree over this cluster (deterministic, different from the launched kernels').
//
// Reductions: each CTA sums its threads' partials (warp shuffles, then warps in order) into
// one of four rotating slots of its shared memory; after the cluster barrier every CTA adds
// all CTAs' slots in rank order and applies the scalar step to its own copy of the scalars,
// so every CTA holds the same scalars and takes the same branches. A slot is written again
// four reductions later, by which time every CTA has read it (three barriers lie between).
// The loop stops at the scalar step's done flag, or after nmax + 2 bodies (info -5), in every
// CTA at the same point; the last barrier keeps every CTA's shared memory alive until all have
// read it.
#pragma once

#include <cooperative_groups.h>

#include "fiim_kernels.cuh"

namespace fiim {

constexpr int kClusterCtas = 16;        // CTAs of the cluster (non-portable size, B200)
constexpr int kClusterThreads = 1024;   // threads per CTA
constexpr int kClusterMaxRows = 2048;   // rows per CTA: 12 vectors of 8 B = 192 KB of shared memory
constexpr int kClusterVecs = 12;        // x, r, r0, p (two buffers), v, s, t, pc, sc, tm, D^-1

struct ClusterArgs {
    CsrView<double> A, G, H;   // full CSR in global memory
    int n, rows;               // rows per CTA (the last CTAs may own fewer, or none)
    double *x;                 // in: the initial guess; out: the solution
    const double *b, *IDv;
    DState *st;                // in: the solve's parameters; out: the final scalars
};

// Shared-memory bytes of one CTA for `rows` rows per CTA: the vectors, four reduction slots,
// the scalars, and the row offsets of A, G and H for the CTA's rows.
constexpr size_t cluster_smem(int rows) {
    return sizeof(double) * ((size_t)kClusterVecs * rows + 16) + sizeof(DState) + 64 +
           sizeof(int) * 3 * ((size_t)rows + 1);
}


namespace cl {
namespace cg = cooperative_groups;

// The owner CTA and local offset of row j. A column outside [0, n) (which no valid matrix
// has) is clamped into the cluster, so that it can never address a CTA that does not exist.
__device__ __forceinline__ void owner_of(int j, int rows, unsigned &owner, int &off) {
    owner = min((unsigned)max(j, 0) / (unsigned)rows, (unsigned)kClusterCtas - 1u);
    off = min(max(j - (int)owner * rows, 0), rows - 1);
}

// Entry `off` of the vector at `vec` (the same shared-memory offset in every CTA) of CTA owner.
__device__ __forceinline__ double ld(const cg::cluster_group &cluster, const double *vec, int off, unsigned owner,
                                     unsigned me) {
    if (owner == me) return vec[off];
    return *cluster.map_shared_rank(vec + off, owner);
}

// One product, a thread per row: the row's rounded products summed left to right in storage
// order (the reference's CSR product, bit for bit), then emit(local row, global row, sum).
// xval(owner, off) gives the gathered vector's entry at a column. rp holds the CTA's rows'
// offsets (local row li: rp[li], rp[li + 1]). The loop is pipelined by one entry: the next
// entry's column and value are loaded while this entry's gather is in flight.
//
// Measured against a CSR-stream form of the same product (each warp loading a group's entries
// coalesced into a stage of shared memory, each lane then summing its row there): at 5
// entries per row a 32-row group does not fit a 128-entry stage, and its two 16-row halves
// cost more than a row per lane (33.1 against 21.0 us per iteration at n = 16,384).
template <class XVal, class Emit>
__device__ __forceinline__ void spmv(const CsrView<double> &M, const int *rp, int lo, int hi, int rows, XVal xval,
                                     Emit emit) {
    for (int li = (int)threadIdx.x; lo + li < hi; li += (int)blockDim.x) {
        double s = 0.0;
        const int e1 = rp[li + 1];
        int e = rp[li];
        int c = 0;
        double v = 0.0;
        if (e < e1) {
            c = __ldg(M.ci + e);
            v = __ldg(M.v + e);
        }
        for (; e < e1; ++e) {
            int cn = 0;
            double vn = 0.0;
            if (e + 1 < e1) {
                cn = __ldg(M.ci + e + 1);
                vn = __ldg(M.v + e + 1);
            }
            unsigned owner;
            int off;
            owner_of(c, rows, owner, off);
            s = __dadd_rn(s, __dmul_rn(v, xval(owner, off)));
            c = cn;
            v = vn;
        }
        emit(li, lo + li, s);
    }
}

template <class F>
__device__ __forceinline__ void local_rows(int lo, int hi, F f) {
    for (int li = (int)threadIdx.x; lo + li < hi; li += (int)blockDim.x) f(li);
}

// The cluster's sums of v (a fixed tree: each warp's lanes, then the CTA's warps in warp 0,
// then the CTAs' sums in warp 0, lane c holding CTA c's), then fin.finish on this CTA's
// scalars. Every step of the tree is a warp's shuffles, so no thread adds a long chain of
// partials (or waits on a chain of remote loads) while the others wait at the barrier.
template <int NR, class Fin>
__device__ __forceinline__ void reduce(const cg::cluster_group &cluster, double (&v)[NR], double *slots, int &slot,
                                       DState *sst, const Fin &fin) {
    __shared__ double sm[kClusterThreads / 32][4];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < NR; ++j) v[j] = warp_sum(v[j]);
    if (lane == 0)
#pragma unroll
        for (int j = 0; j < NR; ++j) sm[w][j] = v[j];
    __syncthreads();
    double *mine = slots + slot * 4;
    if (w == 0) {
#pragma unroll
        for (int j = 0; j < NR; ++j) {
            const double s = warp_sum(lane < (int)(blockDim.x >> 5) ? sm[lane][j] : 0.0);
            if (lane == 0) mine[j] = s;
        }
    }
    cluster.sync();
    if (w == 0) {
        double acc[NR];
#pragma unroll
        for (int j = 0; j < NR; ++j)
            acc[j] = warp_sum(lane < (int)cluster.num_blocks() ? *cluster.map_shared_rank(mine + j, (unsigned)lane) : 0.0);
        if (lane == 0) fin.finish(sst, acc);
    }
    __syncthreads();
    slot = (slot + 1) & 3;
#pragma unroll
    for (int j = 0; j < NR; ++j) v[j] = 0.0;
}

}  // namespace cl

// The first half of the body's scalars in one step: ||pc||^2 (stagnation test), alpha from
// r0 . v (with ACIFIM's guard), ||r||^2 and ||x||^2 (the tests), as EpiNorm, EpiAlpha and
// FinS apply them one by one.
struct FinPcAlphaS {
    __device__ void finish(DState *st, const double *t) const {
        st->pc2 = t[0];
        EpiAlpha{nullptr, nullptr}.finish(st, t + 1);
        FinS{}.finish(st, t + 2);
    }
};

static __global__ void __launch_bounds__(kClusterThreads, 1) k_solve_cluster(ClusterArgs a) {
    namespace cg = cooperative_groups;
    const cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ double csm[];
    const int R = a.rows;
    // Vector k of this CTA's rows starts at csm + k R; the addresses are recomputed where they
    // are used (a base and a kernel argument), which keeps registers free for the loads. p has
    // two buffers: the next p is formed while the current one is still being gathered.
    enum { kX, kR, kR0, kPa, kPb, kV, kS, kT, kPC, kSC, kTM, kD };
#define FIIM_CV(k) (csm + (k) * R)
    double *slots = FIIM_CV(kClusterVecs);
    DState &sst = *reinterpret_cast<DState *>(slots + 16);
#define FIIM_CRP(m) (reinterpret_cast<int *>(reinterpret_cast<char *>(slots + 16) + sizeof(DState) + 64) + (m) * (R + 1))
    const unsigned me = cluster.block_rank();
    const int lo = min(a.n, (int)me * R), hi = min(a.n, lo + R);
    int slot = 0;
    auto vec = [&](int k) { return (const double *)FIIM_CV(k); };
    auto plain = [&](int k) {
        return [&, k](unsigned o, int off) { return cl::ld(cluster, vec(k), off, o, me); };
    };
    cl::local_rows(lo, hi, [&](int li) {
        FIIM_CV(kX)[li] = a.x[lo + li];
        FIIM_CV(kD)[li] = __ldg(a.IDv + lo + li);
    });
    for (int li = (int)threadIdx.x; li <= hi - lo; li += (int)blockDim.x) {
        FIIM_CRP(0)[li] = __ldg(a.A.rp + lo + li);
        FIIM_CRP(1)[li] = __ldg(a.G.rp + lo + li);
        FIIM_CRP(2)[li] = __ldg(a.H.rp + lo + li);
    }
    if (threadIdx.x == 0) sst = *a.st;
    __syncthreads();
    cluster.sync();   // every CTA's x is in place before the first gather
    // Start: r = b - A x, r0 = r, p = r, ro = ||r0|| (AFIIM/src/bicgstab.cpp:151-165).
    {
        double red[1] = {0.0};
        cl::spmv(a.A, FIIM_CRP(0), lo, hi, R, plain(kX), [&](int li, int i, double s) {
            const double pi = __dadd_rn(__ldg(a.b + i), __dmul_rn(-1.0, s));
            FIIM_CV(kPa)[li] = pi;
            FIIM_CV(kR0)[li] = pi;
            FIIM_CV(kR)[li] = pi;
            red[0] += pi * pi;
        });
        cl::reduce<1>(cluster, red, slots, slot, &sst, FinInit{});   // its barrier completes p
    }
    int loops = 0, pcur = kPa;
    for (;;) {
        if (sst.done) break;
        if (++loops > sst.nmax + 2) {   // device-side guard (the scalar steps stop at nmax)
            if (threadIdx.x == 0) sst.info = -5;
            break;
        }
        // tm = D^-1 o (H p). From the second iteration on, p = (-beta omega) v + beta p + r
        // (:270-271) is formed at each gathered entry from r, v and the previous p, rounded as
        // the update rounds it, and this CTA's rows of it go to the other buffer.
        if (loops == 1) {
            cl::spmv(a.H, FIIM_CRP(2), lo, hi, R, plain(pcur),
                     [&](int li, int, double s) { FIIM_CV(kTM)[li] = __dmul_rn(FIIM_CV(kD)[li], s); });
        } else {
            const double bb = sst.beta, c = __dmul_rn(-sst.beta, sst.omega);
            const int pold = pcur, pnew = (pcur == kPa) ? kPb : kPa;
            auto pval = [&](unsigned o, int off) {
                const double vj = cl::ld(cluster, vec(kV), off, o, me), pj = cl::ld(cluster, vec(pold), off, o, me);
                return __dadd_rn(__dadd_rn(__dmul_rn(c, vj), __dmul_rn(bb, pj)), cl::ld(cluster, vec(kR), off, o, me));
            };
            cl::spmv(a.H, FIIM_CRP(2), lo, hi, R, pval,
                     [&](int li, int, double s) { FIIM_CV(kTM)[li] = __dmul_rn(FIIM_CV(kD)[li], s); });
            cl::local_rows(lo, hi, [&](int li) {
                const double pi = __dadd_rn(__dmul_rn(c, FIIM_CV(kV)[li]), __dmul_rn(bb, FIIM_CV(pold)[li]));
                FIIM_CV(pnew)[li] = __dadd_rn(pi, FIIM_CV(kR)[li]);
            });
            pcur = pnew;
        }
        cluster.sync();
        // pc = G tm (||pc||^2); v = A pc (r0 . v); ||r||^2, ||x||^2; alpha (:172-185, :201, :216)
        {
            double red[4] = {0.0, 0.0, 0.0, 0.0};
            cl::spmv(a.G, FIIM_CRP(1), lo, hi, R, plain(kTM), [&](int li, int, double s) {
                FIIM_CV(kPC)[li] = s;
                red[0] += s * s;
            });
            cluster.sync();
            cl::spmv(a.A, FIIM_CRP(0), lo, hi, R, plain(kPC), [&](int li, int, double s) {
                FIIM_CV(kV)[li] = s;
                red[1] += FIIM_CV(kR0)[li] * s;
            });
            cl::local_rows(lo, hi, [&](int li) {
                const double ri = FIIM_CV(kR)[li], xi = FIIM_CV(kX)[li];
                red[2] += ri * ri;
                red[3] += xi * xi;
            });
            cl::reduce<4>(cluster, red, slots, slot, &sst, FinPcAlphaS{});
        }
        if (sst.done) break;   // non-finite alpha (ACIFIM)
        // tm = D^-1 o (H s), with s = r - alpha v (:184-185) formed at each gathered entry as
        // the update rounds it, and this CTA's rows of s stored; sc = G tm; t = A sc, omega
        // (:189-198)
        {
            const double na = -sst.alpha;
            auto sval = [&](unsigned o, int off) {
                return __dadd_rn(cl::ld(cluster, vec(kR), off, o, me), __dmul_rn(na, cl::ld(cluster, vec(kV), off, o, me)));
            };
            cl::spmv(a.H, FIIM_CRP(2), lo, hi, R, sval,
                     [&](int li, int, double s) { FIIM_CV(kTM)[li] = __dmul_rn(FIIM_CV(kD)[li], s); });
            cl::local_rows(lo, hi, [&](int li) {
                FIIM_CV(kS)[li] = __dadd_rn(FIIM_CV(kR)[li], __dmul_rn(na, FIIM_CV(kV)[li]));
            });
            cluster.sync();
            cl::spmv(a.G, FIIM_CRP(1), lo, hi, R, plain(kTM), [&](int li, int, double s) { FIIM_CV(kSC)[li] = s; });
            cluster.sync();
            double red[2] = {0.0, 0.0};
            cl::spmv(a.A, FIIM_CRP(0), lo, hi, R, plain(kSC), [&](int li, int, double s) {
                FIIM_CV(kT)[li] = s;
                red[0] += s * FIIM_CV(kS)[li];
                red[1] += s * s;
            });
            cl::reduce<2>(cluster, red, slots, slot, &sst, EpiOmega{nullptr, nullptr});
        }
        // x += alpha pc + omega sc; r = s - omega t; r0 . r; tests and beta (:207-274)
        {
            double red[1] = {0.0};
            const double al = sst.alpha, om = sst.omega, nom = -sst.omega;
            cl::local_rows(lo, hi, [&](int li) {
                double xi = FIIM_CV(kX)[li];
                xi = __dadd_rn(xi, __dmul_rn(al, FIIM_CV(kPC)[li]));
                xi = __dadd_rn(xi, __dmul_rn(om, FIIM_CV(kSC)[li]));
                FIIM_CV(kX)[li] = xi;
                const double ri = __dadd_rn(FIIM_CV(kS)[li], __dmul_rn(nom, FIIM_CV(kT)[li]));
                FIIM_CV(kR)[li] = ri;
                red[0] += FIIM_CV(kR0)[li] * ri;
            });
            cl::reduce<1>(cluster, red, slots, slot, &sst, FinControl{});   // its barrier completes r
        }
    }
    // FP64 true residual ||b - A x|| / ||b||, then the results for the host.
    cluster.sync();   // x complete in every CTA
    {
        double red[2] = {0.0, 0.0};
        cl::spmv(a.A, FIIM_CRP(0), lo, hi, R, plain(kX), [&](int, int i, double s) {
            const double bi = __ldg(a.b + i), ri = bi - s;
            red[0] += ri * ri;
            red[1] += bi * bi;
        });
        cl::reduce<2>(cluster, red, slots, slot, &sst, EpiResid{nullptr, nullptr});
    }
    cl::local_rows(lo, hi, [&](int li) { a.x[lo + li] = FIIM_CV(kX)[li]; });
    if (me == 0 && threadIdx.x == 0) *a.st = sst;   // one launch: loops stays 0
    cluster.sync();   // no CTA leaves while another may still read its shared memory
#undef FIIM_CV
#undef FIIM_CRP
}

}  // namespace fiim
