// Batched solve: many independent systems in one device-driven loop.
//
// Input: the systems concatenated as one block-diagonal CSR in global numbering (system
// k owns rows and columns [sys_rows[k], sys_rows[k+1])), for A, G, H, and D^-1, b, x.
// Each system runs the reference's loop with its own scalars, divergence window
// (min(max(n_k,500)/50,20), or min(max(n_k,2000)/50,40) for ACIFIM) and termination; a
// finished system's row blocks are skipped. One CUDA graph with a WHILE node runs the
// batched loop body (nine passes plus five per-system finish kernels) until no system is
// active.
//
// Layout: CSR per matrix + row blocks aligned to systems (blk_sys, sys_blk); factor values
// FP64, FP32 or BF16 (fiim_options.precision); A, D^-1 and all vectors FP64; per-system
// state as arrays of nsys entries. Each matrix whose rows allow it also has a sliced-diagonal
// copy with slices inside the systems, which serves its products (FIIM_DIA=0: CSR streams).

#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "fiim_b200.h"
#include "fiim_batch.cuh"
#include "fiim_internal.h"
#include "fiim_kernels.cuh"
#include "fiim_solver.h"

namespace fiim {
namespace {

constexpr int kTile = 2048;

struct BMat {
    DevCsr M;
    int *blk_sys = nullptr, *sys_blk = nullptr;   // device
    int *flag = nullptr;                           // device: finished-system flag per row block
    float *v32 = nullptr;
    __nv_bfloat16 *v16 = nullptr;
    // With a sliced-diagonal copy (M.dia): finished-system flag per slice and each system's
    // first slice (device, one allocation).
    int *sflag = nullptr, *sys_sl = nullptr;
    void *sl_mem = nullptr;
};

// Row blocks per system: consecutive rows of one system, <= max_rows rows, <= tile entries.
void segment_blocks(const std::vector<int> &rp, const std::vector<int> &sys_rows, int tile, int max_rows,
                    std::vector<int> &rb, std::vector<int> &blk_sys, std::vector<int> &sys_blk) {
    rb.assign(1, 0);
    blk_sys.clear();
    sys_blk.assign(1, 0);
    const int nsys = (int)sys_rows.size() - 1;
    for (int k = 0; k < nsys; ++k) {
        int r = sys_rows[k];
        const int end = sys_rows[k + 1];
        while (r < end) {
            if (rp[r + 1] - rp[r] > tile) {
                ++r;
            } else {
                const int start = r;
                long nnz = 0;
                while (r < end && r - start < max_rows && nnz + (rp[r + 1] - rp[r]) <= tile) {
                    nnz += rp[r + 1] - rp[r];
                    ++r;
                }
            }
            rb.push_back(r);
            blk_sys.push_back(k);
        }
        sys_blk.push_back((int)blk_sys.size());
    }
}

template <typename K>
int sgrid(K kernel, long units) { return grid_for(kernel, 1, units); }

}  // namespace

struct BatchSolver : SolverBase {
    BatchSolver() { kind = 0x42415443; }
    int device = -1, nsys = 0, N = 0;
    fiim_options opt{};
    cudaStream_t stream = nullptr;
    Arena arena;
    BMat A, G, H;
    std::vector<int> sys_rows;
    double *IDv = nullptr, *x = nullptr, *b = nullptr, *r = nullptr, *r0 = nullptr, *p = nullptr;
    double *v = nullptr, *sv = nullptr, *t = nullptr, *pc = nullptr, *sc = nullptr, *tm = nullptr;
    double *partials = nullptr;
    bt::BState bs{};
    bt::BGlobal *hg = nullptr;       // pinned host mirror of the global block
    unsigned long long *d_count = nullptr, *h_count = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool host_loop = false;          // FIIM_GRAPH=host: the host relaunches a one-iteration graph
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;

    template <typename V, typename Epi>
    cudaError_t spmv(const BMat &B, const V *vals, const double *xx, const Epi &epi) {
        if (B.M.dia) {   // its sliced-diagonal copy (values of V's width: 2 rows a lane for FP32)
            const DiaView<V> view{B.M.drec, static_cast<const V *>(B.M.dvals), (int)B.M.n, B.M.nsl, B.M.drs};
            if constexpr (sizeof(V) == 8) {
                if (B.M.dsh == 64) {
                    auto k2 = bt::k_bspmv_dia<V, 2, Epi>;
                    return launch_k(k2, grid_for(k2, kWarps, B.M.nsl), 0, stream, view, B.sflag, xx, epi, bs, partials);
                }
                auto k1 = bt::k_bspmv_dia<V, 1, Epi>;
                return launch_k(k1, grid_for(k1, kWarps, B.M.nsl), 0, stream, view, B.sflag, xx, epi, bs, partials);
            } else {
                auto kd = bt::k_bspmv_dia<V, sizeof(V) == 4 ? 2 : 4, Epi>;
                return launch_k(kd, grid_for(kd, kWarps, B.M.nsl), 0, stream, view, B.sflag, xx, epi, bs, partials);
            }
        }
        auto kern = bt::k_bspmv<kTile, V, Epi, false>;
        const int g = sgrid(kern, B.M.nblk);
        if (B.M.narrow) {
            auto kn = bt::k_bspmv<kTile, V, Epi, true>;
            return launch_k(kn, sgrid(kn, B.M.nblk), 0, stream, CsrView<V>{B.M.rp, B.M.ci, vals, (int)B.M.n}, B.M.rb,
                            B.M.eb, B.flag, B.M.nblk, xx, epi, bs, partials, NarrowCols{B.M.cd, B.M.cb});
        }
        return launch_k(kern, g, 0, stream, CsrView<V>{B.M.rp, B.M.ci, vals, (int)B.M.n}, B.M.rb, B.M.eb, B.flag,
                        B.M.nblk, xx, epi, bs, partials, NarrowCols{});
    }
    template <typename Epi>
    cudaError_t spmv_f(const BMat &B, const double *xx, const Epi &epi) {   // factors: stored precision
        if (opt.precision == FIIM_MIXED_BF16) return spmv(B, B.v16, xx, epi);
        if (opt.precision == FIIM_MIXED_FP32) return spmv(B, B.v32, xx, epi);
        return spmv(B, B.M.v, xx, epi);
    }

    // Second phase of a per-system reduction (bt::k_bfinish) after a product with matrix B:
    // over its slices when its sliced-diagonal copy served, else over its row blocks.
    template <int NR, bool GATED = true, class Fin>
    cudaError_t finish(const BMat &B, const Fin &fin) {
        const int g = (int)std::min<long>(nsys, 8L * num_sms());
        if (B.M.dia) return launch_k(bt::k_bfinish<NR, GATED, Fin>, g, 0, stream, B.sys_sl, 1, nsys, partials, bs, fin);
        return launch_k(bt::k_bfinish<NR, GATED, Fin>, g, 0, stream, B.sys_blk, kWarps, nsys, partials, bs, fin);
    }
    // ... after a vector update, which walks A's row blocks.
    template <int NR, class Fin>
    cudaError_t finish_rows(const Fin &fin) {
        const int g = (int)std::min<long>(nsys, 8L * num_sms());
        return launch_k(bt::k_bfinish<NR, true, Fin>, g, 0, stream, A.sys_blk, kWarps, nsys, partials, bs, fin);
    }

    // The sliced-diagonal copy of B (fiim_internal.h, build_dia_structure) with slices inside
    // the systems, its values `vals` (device, the stored width vbytes), its slice flags and the
    // systems' first slices; B keeps its CSR streams when the matrix does not allow it.
    int build_copy(BMat &B, int m, int vbytes, const void *vals) {
        FIIM_TRY(build_dia_structure(B.M, stream, vbytes, &sys_rows));
        if (!B.M.dia_mem) return FIIM_OK;
        FIIM_TRY(place_dia(B.M, vals, stream));
        if (!B.M.dia) return FIIM_OK;
        const size_t bf = Arena::need(sizeof(int) * std::max(B.M.nsl, 1)), bsl = Arena::need(sizeof(int) * (nsys + 1));
        char *mem = nullptr;
        if (cudaMalloc(&mem, bf + bsl) != cudaSuccess) {
            cudaGetLastError();
            release_dia(B.M);   // no room: the CSR streams serve
            return FIIM_OK;
        }
        B.sl_mem = mem;
        B.sflag = reinterpret_cast<int *>(mem);
        B.sys_sl = reinterpret_cast<int *>(mem + bf);
        FIIM_CUDA(cudaMemcpyAsync(B.sys_sl, B.M.hseg_sl.data(), sizeof(int) * (nsys + 1), cudaMemcpyHostToDevice,
                                  stream));
        FIIM_CUDA(cudaStreamSynchronize(stream));
        bs.bf[3 + m] = bt::BlockFlags{B.sflag, B.sys_sl};
        return FIIM_OK;
    }

    int enqueue_iteration(bool cond, cudaGraphConditionalHandle h) {
        const int nb = A.M.nblk;
        FIIM_CUDA(spmv_f(H, p, bt::BEpiScale{tm, IDv}));
        FIIM_CUDA(spmv_f(G, tm, bt::BEpiNorm{pc}));
        FIIM_CUDA(finish<1>(G, bt::BEpiNorm{pc}));
        FIIM_CUDA(spmv(A, A.M.v, pc, bt::BEpiAlpha{v, r0}));
        FIIM_CUDA(finish<1>(A, bt::BEpiAlpha{v, r0}));
        FIIM_CUDA(launch_k(bt::k_bupdate_s, sgrid(bt::k_bupdate_s, nb), 0, stream, A.M.rb, A.blk_sys, A.sys_blk,
                           nb, r, v, x, sv, bs, partials));
        FIIM_CUDA(finish_rows<2>(bt::BFinS{}));
        FIIM_CUDA(spmv_f(H, sv, bt::BEpiScale{tm, IDv}));
        FIIM_CUDA(spmv_f(G, tm, bt::BEpiStore{sc}));
        FIIM_CUDA(spmv(A, A.M.v, sc, bt::BEpiOmega{t, sv}));
        FIIM_CUDA(finish<2>(A, bt::BEpiOmega{t, sv}));
        FIIM_CUDA(launch_k(bt::k_bupdate_xr, sgrid(bt::k_bupdate_xr, nb), 0, stream, A.M.rb, A.blk_sys, A.sys_blk,
                           nb, pc, sc, sv, t, r0, x, r, bs, partials));
        FIIM_CUDA(finish_rows<1>(bt::BFinControl{}));
        FIIM_CUDA(launch_k(bt::k_bupdate_p, sgrid(bt::k_bupdate_p, nb), 0, stream, A.M.rb, A.blk_sys, nb, r, v, p,
                           bs, h, cond ? 1 : 0));
        return FIIM_OK;
    }

    int set_blocks(BMat &B) {
        std::vector<int> rb, bsys, sblk;
        segment_blocks(B.M.hrp, sys_rows, kTile - 1, kThreads, rb, bsys, sblk);   // pairs: <= TILE - 1
        B.M.tile = kTile;
        B.M.nblk = (int)bsys.size();
        std::vector<int> eb(rb.size());
        for (size_t q = 0; q < rb.size(); ++q) eb[q] = B.M.hrp[rb[q]];
        FIIM_CUDA(cudaMemcpyAsync(B.M.rb, rb.data(), sizeof(int) * rb.size(), cudaMemcpyHostToDevice, stream));
        FIIM_CUDA(cudaMemcpyAsync(B.M.eb, eb.data(), sizeof(int) * eb.size(), cudaMemcpyHostToDevice, stream));
        if (!bsys.empty())
            FIIM_CUDA(cudaMemcpyAsync(B.blk_sys, bsys.data(), sizeof(int) * bsys.size(), cudaMemcpyHostToDevice,
                                      stream));
        FIIM_CUDA(cudaMemcpyAsync(B.sys_blk, sblk.data(), sizeof(int) * sblk.size(), cudaMemcpyHostToDevice, stream));
        FIIM_CUDA(cudaStreamSynchronize(stream));
        return build_narrow(B.M, stream);
    }

    int create(int nsys_, const int *sys_rows_, const int *Ai, const int *Aj, const double *Av, const int *Gi,
               const int *Gj, const double *Gv, const double *IDv_, const int *Hi, const int *Hj, const double *Hv,
               const fiim_options &o) {
        opt = o;
        nsys = nsys_;
        if (nsys <= 0 || !sys_rows_ || !Ai || !Aj || !Av || !Gi || !Gj || !Gv || !IDv_ || !Hi || !Hj || !Hv)
            return set_error(FIIM_EARG, "batch needs nsys > 0, sys_rows and A, G, IDv, H");
        if (opt.issym) return set_error(FIIM_EARG, "batch takes general (non-symmetric-storage) input");
        if (opt.variant == FIIM_ACIFIM && opt.mode != 'E')
            return set_error(FIIM_EARG, "batch applies the explicit product (mode 'E')");
        sys_rows.assign(sys_rows_, sys_rows_ + nsys + 1);   // host array in either memory mode
        if (sys_rows[0] != 0) return set_error(FIIM_EARG, "sys_rows[0] must be 0");
        for (int k = 0; k < nsys; ++k)
            if (sys_rows[k + 1] <= sys_rows[k]) return set_error(FIIM_EARG, "system %d is empty or sys_rows decreases", k);
        N = sys_rows[nsys];
        FIIM_TRY(check_device(&device));
        FIIM_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        FIIM_CUDA(cudaEventCreate(&ev0));
        FIIM_CUDA(cudaEventCreate(&ev1));
        const bool dev = (opt.memory == FIIM_MEM_DEVICE);
        auto nnz_of = [&](const int *rp) -> long {
            if (!dev) return rp[N];
            int z = 0;
            if (cudaMemcpy(&z, rp + N, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
            return z;
        };
        const long nA = nnz_of(Ai), nG = nnz_of(Gi), nH = nnz_of(Hi);
        if (nA < 0 || nG < 0 || nH < 0) return set_error(FIIM_ECUDA, "reading row offsets failed");
        // Block-diagonal check (host input): every column inside its row's system.
        if (!dev) {
            const int *rps[3] = {Ai, Gi, Hi};
            const int *cis[3] = {Aj, Gj, Hj};
            for (int m = 0; m < 3; ++m)
                for (int k = 0; k < nsys; ++k)
                    for (int i = sys_rows[k]; i < sys_rows[k + 1]; ++i)
                        for (int q = rps[m][i]; q < rps[m][i + 1]; ++q)
                            if (cis[m][q] < sys_rows[k] || cis[m][q] >= sys_rows[k + 1])
                                return set_error(FIIM_EARG, "matrix %d row %d reaches outside system %d", m, i, k);
        }
        const bool f32 = (opt.precision == FIIM_MIXED_FP32), f16 = (opt.precision == FIIM_MIXED_BF16);
        const size_t vsz = f16 ? 2 : 4;
        size_t bytes = csr_bytes(N, nA) + csr_bytes(N, nG) + csr_bytes(N, nH);
        bytes += 3 * 3 * Arena::need(sizeof(int) * (N + nsys + 1));        // blk_sys, sys_blk, flag
        if (f32 || f16) bytes += Arena::need(vsz * std::max<long>(nG, 1)) + Arena::need(vsz * std::max<long>(nH, 1));
        bytes += 12 * Arena::need(sizeof(double) * N);
        bytes += 12 * Arena::need(sizeof(double) * nsys) + 7 * Arena::need(sizeof(int) * nsys);
        bytes += Arena::need(sizeof(bt::BGlobal)) + 4096;
        FIIM_TRY(arena.reserve(bytes));
        BMat *mats[3] = {&A, &G, &H};
        const long nz[3] = {nA, nG, nH};
        for (int m = 0; m < 3; ++m) {
            FIIM_TRY(carve_csr(arena, mats[m]->M, N, nz[m]));
            mats[m]->blk_sys = static_cast<int *>(arena.take(sizeof(int) * (N + nsys + 1)));
            mats[m]->sys_blk = static_cast<int *>(arena.take(sizeof(int) * (N + nsys + 1)));
            mats[m]->flag = static_cast<int *>(arena.take(sizeof(int) * (N + nsys + 1)));
            if (!mats[m]->blk_sys || !mats[m]->sys_blk || !mats[m]->flag)
                return set_error(FIIM_ENOMEM, "arena exhausted");
            bs.bf[m] = bt::BlockFlags{mats[m]->flag, mats[m]->sys_blk};
        }
        for (int m = 1; m < 3 && (f32 || f16); ++m) {
            void *pv = arena.take(vsz * std::max<long>(nz[m], 1));
            if (!pv) return set_error(FIIM_ENOMEM, "arena exhausted");
            if (f16) mats[m]->v16 = static_cast<__nv_bfloat16 *>(pv);
            else mats[m]->v32 = static_cast<float *>(pv);
        }
        double **vecs[] = {&IDv, &x, &b, &r, &r0, &p, &v, &sv, &t, &pc, &sc, &tm};
        for (auto pp : vecs)
            if (!(*pp = static_cast<double *>(arena.take(sizeof(double) * N)))) return set_error(FIIM_ENOMEM, "arena");
        double **ds[] = {&bs.ro, &bs.rc, &bs.m1, &bs.m2, &bs.alpha, &bs.omega, &bs.beta, &bs.pc2, &bs.x2, &bs.r2,
                         &bs.ts, &bs.tt};
        for (auto pp : ds)
            if (!(*pp = static_cast<double *>(arena.take(sizeof(double) * nsys)))) return set_error(FIIM_ENOMEM, "arena");
        int **is[] = {&bs.iter, &bs.stag, &bs.msteps, &bs.maxmsteps, &bs.info, &bs.done};
        for (auto pp : is)
            if (!(*pp = static_cast<int *>(arena.take(sizeof(int) * nsys)))) return set_error(FIIM_ENOMEM, "arena");
        bs.g = static_cast<bt::BGlobal *>(arena.take(sizeof(bt::BGlobal)));
        d_count = static_cast<unsigned long long *>(arena.take(sizeof(unsigned long long)));
        if (!bs.g || !d_count) return set_error(FIIM_ENOMEM, "arena exhausted");
        FIIM_CUDA(cudaHostAlloc(&hg, sizeof(bt::BGlobal) + 64, cudaHostAllocDefault));
        h_count = reinterpret_cast<unsigned long long *>(reinterpret_cast<char *>(hg) + sizeof(bt::BGlobal) + 32);

        FIIM_TRY(upload_csr(A.M, nA, N, Ai, Aj, Av, 0, dev, stream, d_count, h_count));
        FIIM_TRY(upload_csr(G.M, nG, N, Gi, Gj, Gv, 1, dev, stream, d_count, h_count));
        FIIM_TRY(upload_csr(H.M, nH, N, Hi, Hj, Hv, 2, dev, stream, d_count, h_count));
        FIIM_CUDA(cudaMemcpyAsync(IDv, IDv_, sizeof(double) * N, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                  stream));
        for (int m = 1; m < 3; ++m) {
            const long c = mats[m]->M.nnz;
            if (c <= 0) continue;
            if (f32) bt::k_vals_to_f32<<<grid_for(bt::k_vals_to_f32, kThreads, c), kThreads, 0, stream>>>(
                c, mats[m]->M.v, mats[m]->v32);
            if (f16) mx_to_bf16(mats[m]->M.v, mats[m]->v16, c);
            FIIM_CUDA(cudaGetLastError());
        }
        for (int m = 0; m < 3; ++m) FIIM_TRY(set_blocks(*mats[m]));
        // Sliced-diagonal copies where the matrices allow them: A in FP64, G and H in the
        // factors' stored precision.
        const int fvb = f16 ? 2 : (f32 ? 4 : 8);
        FIIM_TRY(build_copy(A, 0, 8, A.M.v));
        FIIM_TRY(build_copy(G, 1, fvb, f16 ? (const void *)G.v16 : f32 ? (const void *)G.v32 : (const void *)G.M.v));
        FIIM_TRY(build_copy(H, 2, fvb, f16 ? (const void *)H.v16 : f32 ? (const void *)H.v32 : (const void *)H.M.v));
        // Partials of the largest count: per warp of a row block, or per slice (two values each).
        long maxq = std::max({(long)A.M.nblk, (long)G.M.nblk, (long)H.M.nblk, 1L}) * kWarps;
        for (const BMat *B : {&A, &G, &H}) maxq = std::max(maxq, (long)B->M.nsl);
        FIIM_CUDA(cudaMalloc(&partials, sizeof(double) * 2 * maxq));
        // per-system divergence windows (AFIIM/src/bicgstab.cpp:114, ACIFIM/src/bicgstab.cpp:132)
        std::vector<int> mm(nsys);
        for (int k = 0; k < nsys; ++k) {
            const int nk = sys_rows[k + 1] - sys_rows[k];
            mm[k] = (opt.variant == FIIM_ACIFIM) ? std::min(std::max(nk, 2000) / 50, 40)
                                                 : std::min(std::max(nk, 500) / 50, 20);
        }
        FIIM_CUDA(cudaMemcpyAsync(bs.maxmsteps, mm.data(), sizeof(int) * nsys, cudaMemcpyHostToDevice, stream));
        FIIM_CUDA(cudaStreamSynchronize(stream));
        return build_graph();
    }

    void mx_to_bf16(const double *in, __nv_bfloat16 *out, long c);

    int reset_state(double tol, int nmax) {
        bt::BGlobal g = {};
        g.tol = tol;
        g.eps = 1.11022302462516e-16;
        g.nmax = nmax;
        g.alpha_guard = (opt.variant == FIIM_ACIFIM);
        g.active = nsys;
        g.loops = 0;
        g.loops_total = 0;
        *hg = g;
        FIIM_CUDA(cudaMemcpyAsync(bs.g, hg, sizeof(bt::BGlobal), cudaMemcpyHostToDevice, stream));
        FIIM_CUDA(cudaMemsetAsync(bs.done, 0, sizeof(int) * nsys, stream));
        FIIM_CUDA(cudaMemsetAsync(bs.info, 0xff, sizeof(int) * nsys, stream));   // -1
        for (const BMat *B : {&A, &G, &H}) {
            FIIM_CUDA(cudaMemsetAsync(B->flag, 0, sizeof(int) * std::max(B->M.nblk, 1), stream));
            if (B->sflag) FIIM_CUDA(cudaMemsetAsync(B->sflag, 0, sizeof(int) * std::max(B->M.nsl, 1), stream));
        }
        return FIIM_OK;
    }

    int build_graph() {
        // Resolve launch shapes outside capture with every system marked done.
        FIIM_TRY(reset_state(0.0, 0));
        std::vector<int> ones(nsys, 1);
        FIIM_CUDA(cudaMemcpyAsync(bs.done, ones.data(), sizeof(int) * nsys, cudaMemcpyHostToDevice, stream));
        for (const BMat *B : {&A, &G, &H}) {   // nonzero: finished
            FIIM_CUDA(cudaMemsetAsync(B->flag, 1, sizeof(int) * std::max(B->M.nblk, 1), stream));
            if (B->sflag) FIIM_CUDA(cudaMemsetAsync(B->sflag, 1, sizeof(int) * std::max(B->M.nsl, 1), stream));
        }
        FIIM_TRY(enqueue_iteration(false, cudaGraphConditionalHandle{}));
        FIIM_CUDA(cudaStreamSynchronize(stream));
        // FIIM_GRAPH=host: a graph of one loop iteration, relaunched by the host (the same
        // kernels and shapes; for profilers that replay graph kernel nodes one by one).
        const char *mode_env = std::getenv("FIIM_GRAPH");
        if (mode_env && std::strcmp(mode_env, "host") == 0) {
            FIIM_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            const int rc = enqueue_iteration(false, cudaGraphConditionalHandle{});
            cudaGraph_t g1 = nullptr;
            const cudaError_t ec = cudaStreamEndCapture(stream, &g1);
            if (rc != FIIM_OK) return rc;
            FIIM_CUDA(ec);
            FIIM_CUDA(cudaGraphInstantiate(&exec, g1, 0));
            graph = g1;
            host_loop = true;
            return FIIM_OK;
        }
        cudaGraph_t g = nullptr;
        FIIM_CUDA(cudaGraphCreate(&g, 0));
        cudaGraphConditionalHandle h;
        FIIM_CUDA(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        FIIM_CUDA(cudaGraphAddNode(&node, g, nullptr, 0, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        FIIM_CUDA(cudaStreamBeginCaptureToGraph(stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        const int rc = enqueue_iteration(true, h);
        cudaGraph_t captured = nullptr;
        const cudaError_t ec = cudaStreamEndCapture(stream, &captured);
        if (rc != FIIM_OK) return rc;
        FIIM_CUDA(ec);
        FIIM_CUDA(cudaGraphInstantiate(&exec, g, 0));
        graph = g;
        return FIIM_OK;
    }

    // The loop until no system is active: the WHILE graph, or (FIIM_GRAPH=host) a one-body
    // graph relaunched by the host.
    int run_loop(int nmax) {
        if (!host_loop) {
            FIIM_CUDA(cudaGraphLaunch(exec, stream));
            return FIIM_OK;
        }
        int launched = 0, chunk = 1;
        for (;;) {
            for (int q = 0; q < chunk; ++q) FIIM_CUDA(cudaGraphLaunch(exec, stream));
            launched += chunk;
            FIIM_CUDA(cudaMemcpyAsync(hg, bs.g, sizeof(bt::BGlobal), cudaMemcpyDeviceToHost, stream));
            FIIM_CUDA(cudaStreamSynchronize(stream));
            if (hg->active <= 0) break;
            if (launched > std::max(nmax, 0) + 2)
                return set_error(FIIM_ETIMEOUT, "batch not finished after %d iterations", launched);
            chunk = std::min(chunk * 2, 16);
        }
        hg->loops = launched;
        FIIM_CUDA(cudaMemcpyAsync(&bs.g->loops, &hg->loops, sizeof(int), cudaMemcpyHostToDevice, stream));
        return FIIM_OK;
    }

    int solve(const double *b_in, double *x_io, double tol, int nmax, int *iter, int *info, double *resval,
              double *true_relres, fiim_result *summary) {
        FIIM_CUDA(cudaSetDevice(device));
        const bool dev = (opt.memory == FIIM_MEM_DEVICE);
        const cudaMemcpyKind kin = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        FIIM_CUDA(cudaEventRecord(ev0, stream));
        FIIM_CUDA(cudaMemcpyAsync(b, b_in, sizeof(double) * N, kin, stream));
        FIIM_CUDA(cudaMemcpyAsync(x, x_io, sizeof(double) * N, kin, stream));
        FIIM_TRY(reset_state(tol, nmax));
        FIIM_CUDA(spmv(A, A.M.v, x, bt::BEpiInit{b, p, r0, r}));
        FIIM_CUDA(finish<1>(A, bt::BEpiInit{b, p, r0, r}));
        FIIM_TRY(run_loop(nmax));
        FIIM_CUDA(spmv(A, A.M.v, x, bt::BEpiResid{b}));
        FIIM_CUDA((finish<2, false>(A, bt::BEpiResid{b})));
        // Verified: systems whose FP64 true residual misses the target restart from their
        // current x (the others stay finished), until none misses or the rounds run out.
        int rounds = 0, extra = 0;   // restart rounds; launches outside the loop bodies
        while (opt.verified && rounds < opt.max_restarts) {
            ++extra;
            bt::k_bverify<<<std::max(1, std::min((nsys + kThreads - 1) / kThreads, num_sms())), kThreads, 0, stream>>>(
                nsys, bs);
            FIIM_CUDA(cudaGetLastError());
            FIIM_CUDA(cudaMemcpyAsync(hg, bs.g, sizeof(bt::BGlobal), cudaMemcpyDeviceToHost, stream));
            FIIM_CUDA(cudaStreamSynchronize(stream));
            if (hg->active < 0) return set_error(FIIM_ETIMEOUT, "device loop guard tripped");
            if (hg->active == 0) break;
            ++rounds;
            extra += 4;
            FIIM_CUDA(spmv(A, A.M.v, x, bt::BEpiRestart{{b, p, r0, r}}));
            FIIM_CUDA(finish<1>(A, bt::BEpiRestart{{b, p, r0, r}}));
            FIIM_TRY(run_loop(nmax));
            FIIM_CUDA(spmv(A, A.M.v, x, bt::BEpiResid{b}));
            FIIM_CUDA((finish<2, false>(A, bt::BEpiResid{b})));
        }
        FIIM_CUDA(cudaMemcpyAsync(x_io, x, sizeof(double) * N, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                  stream));
        FIIM_CUDA(cudaEventRecord(ev1, stream));
        std::vector<int> hit(nsys), hinfo(nsys);
        std::vector<double> hrc(nsys), hro(nsys), hts(nsys), htt(nsys);
        FIIM_CUDA(cudaMemcpyAsync(hit.data(), bs.iter, sizeof(int) * nsys, cudaMemcpyDeviceToHost, stream));
        FIIM_CUDA(cudaMemcpyAsync(hinfo.data(), bs.info, sizeof(int) * nsys, cudaMemcpyDeviceToHost, stream));
        FIIM_CUDA(cudaMemcpyAsync(hrc.data(), bs.rc, sizeof(double) * nsys, cudaMemcpyDeviceToHost, stream));
        FIIM_CUDA(cudaMemcpyAsync(hro.data(), bs.ro, sizeof(double) * nsys, cudaMemcpyDeviceToHost, stream));
        FIIM_CUDA(cudaMemcpyAsync(hts.data(), bs.ts, sizeof(double) * nsys, cudaMemcpyDeviceToHost, stream));
        FIIM_CUDA(cudaMemcpyAsync(htt.data(), bs.tt, sizeof(double) * nsys, cudaMemcpyDeviceToHost, stream));
        FIIM_CUDA(cudaMemcpyAsync(hg, bs.g, sizeof(bt::BGlobal), cudaMemcpyDeviceToHost, stream));
        FIIM_CUDA(cudaStreamSynchronize(stream));
        if (hg->active < 0) return set_error(FIIM_ETIMEOUT, "device loop guard tripped");
        float ms = 0.f;
        FIIM_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
        int maxit = 0, worst = 0;
        double worst_rel = 0.0;
        for (int k = 0; k < nsys; ++k) {
            if (iter) iter[k] = hit[k];
            if (info) info[k] = hinfo[k];
            if (resval) resval[k] = hrc[k] / hro[k];
            const double tr = std::sqrt(hts[k]) / std::sqrt(htt[k]);
            if (true_relres) true_relres[k] = tr;
            maxit = std::max(maxit, hit[k]);
            worst = std::max(worst, hinfo[k]);
            worst_rel = std::max(worst_rel, tr);
        }
        if (summary) {
            summary->iter = maxit;
            summary->info = worst;
            summary->resval = 0.0;
            summary->true_relres = worst_rel;
            summary->refine_steps = rounds;
            summary->device_ms = ms;
            summary->launches = 4 + extra + (hg->loops_total + hg->loops) * 14;
        }
        return FIIM_OK;
    }

    void destroy() {
        if (device >= 0) cudaSetDevice(device);
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
        if (hg) cudaFreeHost(hg);
        if (partials) cudaFree(partials);
        partials = nullptr;
        for (BMat *B : {&A, &G, &H}) {
            if (B->sl_mem) cudaFree(B->sl_mem);
            B->sl_mem = nullptr;
            B->sflag = B->sys_sl = nullptr;
            release_dia(B->M);
        }
        exec = nullptr;
        graph = nullptr;
        ev0 = ev1 = nullptr;
        stream = nullptr;
        hg = nullptr;
        arena.release();
    }
};

static __global__ void k_bvals_to_bf16(long n, const double *__restrict__ in, __nv_bfloat16 *__restrict__ out) {
    FIIM_FOR_ROWS(i, n) { out[i] = __double2bfloat16(in[i]); }
}

void BatchSolver::mx_to_bf16(const double *in, __nv_bfloat16 *out, long c) {
    k_bvals_to_bf16<<<grid_for(k_bvals_to_bf16, kThreads, c), kThreads, 0, stream>>>(c, in, out);
}

}  // namespace fiim

extern "C" {

int fiim_batch_create(fiim_batch_t *out, int nsys, const int *sys_rows, const int *Ai, const int *Aj,
                      const double *Av, const int *Gi, const int *Gj, const double *Gv, const double *IDv,
                      const int *Hi, const int *Hj, const double *Hv, const fiim_options *opt) {
    if (!out) return fiim::set_error(FIIM_EARG, "out is NULL");
    *out = nullptr;
    fiim_options o;
    if (opt) o = *opt;
    else fiim_options_default(&o);
    auto *s = new fiim::BatchSolver;
    const int rc = s->create(nsys, sys_rows, Ai, Aj, Av, Gi, Gj, Gv, IDv, Hi, Hj, Hv, o);
    if (rc != FIIM_OK) {
        s->destroy();
        delete s;
        return rc;
    }
    *out = reinterpret_cast<fiim_batch_t>(s);
    return FIIM_OK;
}

int fiim_batch_solve(fiim_batch_t h, const double *b, double *x, double tol, int NMAX, int *iter, int *info,
                     double *resval, double *true_relres, fiim_result *summary) {
    if (!h || !b || !x) return fiim::set_error(FIIM_EARG, "null argument");
    return reinterpret_cast<fiim::BatchSolver *>(h)->solve(b, x, tol, NMAX, iter, info, resval, true_relres,
                                                             summary);
}

int fiim_batch_destroy(fiim_batch_t h) {
    if (!h) return FIIM_OK;
    auto *s = reinterpret_cast<fiim::BatchSolver *>(h);
    s->destroy();
    delete s;
    return FIIM_OK;
}

}  // extern "C"
