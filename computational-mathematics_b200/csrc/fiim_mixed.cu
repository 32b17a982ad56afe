// Mixed-precision solve: an FP32 BiCGSTAB whose residual the FP64 b - A x replaces (reliable
// updates, the default), or FP64 iterative refinement around an FP32 inner BiCGSTAB.
//
// Layout in HBM (one arena):
//   A   : int32 rp/ci shared by an FP64 value array (outer residual) and an FP32 copy
//         (inner products); row blocks for the CSR-stream kernels.
//   G, H: int32 rp/ci + FP32 values (FIIM_MIXED_FP32) or BF16 values (FIIM_MIXED_BF16).
//   D^-1: FP32.  Outer vectors x, b, r64: FP64.  Inner vectors e, r, r0, p, v, s, t, pc,
//   sc, tm: FP32.  Two DState blocks (inner, outer) and the reduction partials.
// The FP64 factor values are staged through one scratch buffer at set-up and not kept.
//
// Reliable updates (opt.reliable = delta > 0): r64 = b - A x0 (FP64), sigma = ||r64||; one
// FP32 BiCGSTAB on r64 / sigma from e = 0 (the reference's control flow, in one CUDA graph
// with a device-driven WHILE node); its body ends in an IF node that, when the recurrence
// residual has fallen below delta times its running maximum or has met the target, moves
// sigma e into x and replaces r by (b - A x) / sigma (fiim_mixed.cuh, RState). The solve
// stops when that FP64 residual meets tol ||b||; the host reads the scalars once per solve.
//
// Refinement (opt.reliable = 0): r64 = b - A x (FP64, true residual); while ||r64|| >
// tol ||b||: inner BiCGSTAB on r64/||r64|| from e = 0 to inner_tol (the same graph without
// the IF node), x += ||r64|| e, r64 = b - A x. The host reads two scalars per refinement
// step.

#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <vector>

#include "fiim_b200.h"
#include "fiim_internal.h"
#include "fiim_kernels.cuh"
#include "fiim_mixed.cuh"
#include "fiim_solver.h"

namespace fiim {
namespace {

CsrView<double> view64(const DevCsr &M) { return CsrView<double>{M.rp, M.ci, M.v, (int)M.n}; }

template <int TILE, typename V, typename Epi>
cudaError_t rows_f(cudaStream_t s, const DevCsr &M, const V *vals, const float *x, const Epi &epi,
                   DState *st, double *partials) {
    if (M.narrow) {
        auto kern = mx::k_spmv_rows_f<TILE, V, Epi, true>;
        const int g = grid_for(kern, 1, M.nblk);
        return launch_k(kern, g, 0, s, CsrView<V>{M.rp, M.ci, vals, (int)M.n}, M.rb, M.eb, M.nblk, x, epi, st,
                        partials, NarrowCols{M.cd, M.cb});
    }
    auto kern = mx::k_spmv_rows_f<TILE, V, Epi, false>;
    const int g = grid_for(kern, 1, M.nblk);
    return launch_k(kern, g, 0, s, CsrView<V>{M.rp, M.ci, vals, (int)M.n}, M.rb, M.eb, M.nblk, x, epi, st,
                    partials, NarrowCols{});
}

template <typename V, typename Epi>
cudaError_t spmv_f(const DevCsr &M, const V *vals, cudaStream_t s, const float *x, const Epi &epi,
                   DState *st, double *partials) {
    if (M.dia && M.dvbytes == (int)sizeof(V)) {   // the sliced-diagonal copy of these values
        if (M.dseg) return cudaErrorInvalidValue;     // k_spmv_dia takes slices of one segment
        const DiaView<V> view{M.drec, static_cast<const V *>(M.dvals), (int)M.n, M.nsl, M.drs};
        auto kern = k_spmv_dia<V, float, sizeof(V) == 4 ? 2 : 4, Epi>;   // the rows a lane it was built for
        return launch_k(kern, grid_for(kern, kWarps, M.nsl), 0, s, view, x, epi, st, partials);
    }
    switch (M.tile) {
        case 1024: return rows_f<1024>(s, M, vals, x, epi, st, partials);
        case 4096: return rows_f<4096>(s, M, vals, x, epi, st, partials);
        default: return rows_f<2048>(s, M, vals, x, epi, st, partials);
    }
}

template <int TILE, typename Epi>
cudaError_t rows_64(cudaStream_t s, const DevCsr &M, const double *x, const Epi &epi, DState *st,
                    double *partials) {
    auto kern = k_spmv_rows<TILE, Epi, false>;
    const int g = grid_for(kern, 1, M.nblk);
    kern<<<g, kThreads, 0, s>>>(view64(M), M.rb, M.eb, M.nblk, x, epi, st, partials, NarrowCols{});
    return cudaGetLastError();
}

// FP64 product with A (outer residual); the row blocks were built for M.tile.
template <typename Epi>
cudaError_t spmv_64(const DevCsr &M, cudaStream_t s, const double *x, const Epi &epi, DState *st,
                    double *partials) {
    switch (M.tile) {
        case 1024: return rows_64<1024>(s, M, x, epi, st, partials);
        case 4096: return rows_64<4096>(s, M, x, epi, st, partials);
        default: return rows_64<2048>(s, M, x, epi, st, partials);
    }
}

template <typename K>
int sgrid(K kernel, long n) { return grid_for(kernel, kThreads, n); }

}  // namespace

struct MixedSolver : SolverBase {
    MixedSolver() { kind = kKindMixed; }
    int device = -1, n = 0;
    fiim_options opt{};
    bool bf16 = false;
    cudaStream_t stream = nullptr;
    Arena arena;
    DevCsr A, G, H;
    float *A32 = nullptr, *G32 = nullptr, *H32 = nullptr, *D32 = nullptr;
    __nv_bfloat16 *G16 = nullptr, *H16 = nullptr;
    double *x = nullptr, *b = nullptr, *r64 = nullptr, *stage = nullptr;
    float *e = nullptr, *r = nullptr, *r0 = nullptr, *p = nullptr, *v = nullptr, *s = nullptr;
    float *t = nullptr, *pc = nullptr, *sc = nullptr, *tm = nullptr;
    DState *st = nullptr, *sto = nullptr, *hst = nullptr;
    mx::RState *rs = nullptr, *hrs = nullptr;   // reliable updates (device, pinned host copy)
    bool reliable = false;
    double *partials = nullptr;
    unsigned long long *d_count = nullptr, *h_count = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool host_loop = false;   // FIIM_GRAPH=host: the host relaunches a one-iteration inner graph
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;

    template <typename Epi>
    cudaError_t spmv_gh(const DevCsr &M, bool is_g, const float *xx, const Epi &epi) {
        if (bf16) return spmv_f(M, is_g ? G16 : H16, stream, xx, epi, st, partials);
        return spmv_f(M, is_g ? G32 : H32, stream, xx, epi, st, partials);
    }

    // cond: bit 0 = set the WHILE node's condition (hw), bit 1 = set the IF node's (hif,
    // reliable updates); 0 outside a graph.
    int enqueue_inner(int cond, cudaGraphConditionalHandle hw, cudaGraphConditionalHandle hif) {
        const long nn = n;
        FIIM_CUDA(spmv_gh(H, false, p, mx::EpiScaleF{tm, D32}));
        FIIM_CUDA(spmv_gh(G, true, tm, mx::EpiNormF{pc}));
        FIIM_CUDA(spmv_f(A, A32, stream, pc, mx::EpiAlphaF{v, r0}, st, partials));
        FIIM_CUDA(launch_k(mx::k_update_s_f, sgrid(mx::k_update_s_f, nn), 0, stream, nn, r, v, e, s, st, partials));
        FIIM_CUDA(spmv_gh(H, false, s, mx::EpiScaleF{tm, D32}));
        FIIM_CUDA(spmv_gh(G, true, tm, mx::EpiStoreF{sc}));
        FIIM_CUDA(spmv_f(A, A32, stream, sc, mx::EpiOmegaF{t, s}, st, partials));
        if (reliable) {
            auto kxr = mx::k_update_xr_f<mx::FinControlR>;
            FIIM_CUDA(launch_k(kxr, sgrid(kxr, nn), 0, stream, nn, pc, sc, s, t, r0, e, r, st, partials,
                               mx::FinControlR{rs}));
            FIIM_CUDA(launch_k(mx::k_update_p_r, sgrid(mx::k_update_p_r, nn), 0, stream, nn, r, v, p, st,
                               (const mx::RState *)rs, hw, hif, cond));
            return FIIM_OK;
        }
        auto kxr = mx::k_update_xr_f<FinControl>;
        FIIM_CUDA(launch_k(kxr, sgrid(kxr, nn), 0, stream, nn, pc, sc, s, t, r0, e, r, st, partials, FinControl{}));
        FIIM_CUDA(launch_k(mx::k_update_p_f, sgrid(mx::k_update_p_f, nn), 0, stream, nn, r, v, p, st, hw,
                           (cond & 1) ? 1 : 0));
        return FIIM_OK;
    }

    // The replacement of reliable updates (the IF node's body): x += sigma e, e = 0, then
    // r = (b - A x) / sigma with the FP64 A, p moved by the change in r, m1 = r0 . r.
    int enqueue_replace() {
        const long nn = n;
        FIIM_CUDA(launch_k(mx::k_replace_x, sgrid(mx::k_replace_x, nn), 0, stream, nn, e, x,
                           (const mx::RState *)rs));
        FIIM_CUDA(spmv_64(A, stream, x, mx::EpiReplace{b, r, p, r0, rs}, st, partials));
        return FIIM_OK;
    }

    // Captures one inner iteration into `into`; with reliable updates an IF node (hif) that
    // runs the replacement follows the last kernel.
    int capture_body(cudaGraph_t into, int cond, cudaGraphConditionalHandle hw, cudaGraphConditionalHandle hif) {
        FIIM_CUDA(cudaStreamBeginCaptureToGraph(stream, into, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue_inner(cond, hw, hif);
        cudaGraph_t ifbody = nullptr;
        if (rc == FIIM_OK && reliable) {
            cudaStreamCaptureStatus cs;
            const cudaGraphNode_t *deps = nullptr;
            size_t nd = 0;
            cudaGraphNodeParams ip = {};
            ip.type = cudaGraphNodeTypeConditional;
            ip.conditional.handle = hif;
            ip.conditional.type = cudaGraphCondTypeIf;
            ip.conditional.size = 1;
            cudaGraphNode_t ifn;
            cudaError_t ce = cudaStreamGetCaptureInfo(stream, &cs, nullptr, nullptr, &deps, &nd);
            if (ce == cudaSuccess) ce = cudaGraphAddNode(&ifn, into, deps, nd, &ip);
            if (ce == cudaSuccess) ce = cudaStreamUpdateCaptureDependencies(stream, &ifn, 1, cudaStreamSetCaptureDependencies);
            if (ce == cudaSuccess) ifbody = ip.conditional.phGraph_out[0];
            else rc = set_error(FIIM_ECUDA, cudaGetErrorString(ce));
        }
        cudaGraph_t captured = nullptr;
        const cudaError_t ec = cudaStreamEndCapture(stream, &captured);
        if (rc != FIIM_OK) return rc;
        FIIM_CUDA(ec);
        if (!ifbody) return FIIM_OK;
        FIIM_CUDA(cudaStreamBeginCaptureToGraph(stream, ifbody, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        rc = enqueue_replace();
        const cudaError_t ec2 = cudaStreamEndCapture(stream, &captured);
        if (rc != FIIM_OK) return rc;
        FIIM_CUDA(ec2);
        return FIIM_OK;
    }

    int build_graph() {
        // Resolve launch shapes outside capture (every kernel returns at once: done = 1).
        DState hd = {};
        hd.done = 1;
        *hst = hd;
        FIIM_CUDA(cudaMemcpyAsync(st, hst, sizeof(DState), cudaMemcpyHostToDevice, stream));
        FIIM_TRY(enqueue_inner(0, cudaGraphConditionalHandle{}, cudaGraphConditionalHandle{}));
        if (reliable) FIIM_TRY(enqueue_replace());   // writes only this solver's scratch vectors
        FIIM_CUDA(cudaStreamSynchronize(stream));
        // FIIM_GRAPH=host: a graph of one inner iteration, relaunched by the host (the same
        // kernels and shapes; for profilers that replay graph kernel nodes one by one).
        const char *mode_env = std::getenv("FIIM_GRAPH");
        if (mode_env && std::strcmp(mode_env, "host") == 0) {
            cudaGraph_t g1 = nullptr;
            FIIM_CUDA(cudaGraphCreate(&g1, 0));
            graph = g1;
            cudaGraphConditionalHandle hif{};
            if (reliable) FIIM_CUDA(cudaGraphConditionalHandleCreate(&hif, g1, 0, cudaGraphCondAssignDefault));
            FIIM_TRY(capture_body(g1, reliable ? 2 : 0, cudaGraphConditionalHandle{}, hif));
            FIIM_CUDA(cudaGraphInstantiate(&exec, g1, 0));
            host_loop = true;
            return FIIM_OK;
        }
        cudaGraph_t g = nullptr;
        FIIM_CUDA(cudaGraphCreate(&g, 0));
        graph = g;
        cudaGraphConditionalHandle h, hif{};
        FIIM_CUDA(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
        if (reliable) FIIM_CUDA(cudaGraphConditionalHandleCreate(&hif, g, 0, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        FIIM_CUDA(cudaGraphAddNode(&node, g, nullptr, 0, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        FIIM_TRY(capture_body(body, reliable ? 3 : 1, h, hif));
        FIIM_CUDA(cudaGraphInstantiate(&exec, g, 0));
        return FIIM_OK;
    }

    // Tune the FP32 kernels' row-block size per matrix (speed only).
    template <typename V>
    int tune(DevCsr &M, const V *vals) {
        const int cands[3] = {1024, 2048, 4096};
        int best = 2048;
        float best_ms = 1e30f;
        FIIM_CUDA(cudaMemsetAsync(tm, 0, sizeof(float) * n, stream));
        for (int c : cands) {
            FIIM_TRY(set_tile(M, c, stream));
            FIIM_CUDA(spmv_f(M, vals, stream, tm, mx::EpiStoreF{t}, nullptr, nullptr));
            FIIM_CUDA(cudaEventRecord(ev0, stream));
            for (int k = 0; k < 5; ++k) FIIM_CUDA(spmv_f(M, vals, stream, tm, mx::EpiStoreF{t}, nullptr, nullptr));
            FIIM_CUDA(cudaEventRecord(ev1, stream));
            FIIM_CUDA(cudaEventSynchronize(ev1));
            float ms = 0.f;
            FIIM_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
            if (ms < best_ms * 0.97f) {
                best_ms = ms;
                best = c;
            }
        }
        return set_tile(M, best, stream);
    }

    int create(int n_, const int *Ai, const int *Aj, const double *Av, const int *Gi, const int *Gj,
               const double *Gv, const double *IDv, const int *Hi, const int *Hj, const double *Hv,
               const fiim_options &o) {
        opt = o;
        n = n_;
        bf16 = (opt.precision == FIIM_MIXED_BF16);
        if (n <= 0 || !Ai || !Aj || !Av || !Gi || !Gj || !Gv || !IDv || !Hi || !Hj || !Hv)
            return set_error(FIIM_EARG, "mixed precision needs A, G, IDv and H");
        if (opt.issym) return set_error(FIIM_EARG, "mixed precision takes general (non-symmetric-storage) input");
        if (opt.variant == FIIM_ACIFIM && opt.mode != 'E')
            return set_error(FIIM_EARG, "mixed precision applies the explicit product (mode 'E')");
        if (!(opt.inner_tol > 0.0) || opt.inner_nmax <= 0 || opt.max_refine <= 0)
            return set_error(FIIM_EARG, "inner_tol > 0, inner_nmax > 0 and max_refine > 0 are required");
        if (!(opt.reliable >= 0.0 && opt.reliable < 1.0))
            return set_error(FIIM_EARG, "reliable must be 0 (refinement) or a delta in (0, 1)");
        reliable = opt.reliable > 0.0;
        FIIM_TRY(check_device(&device));
        FIIM_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        FIIM_CUDA(cudaEventCreate(&ev0));
        FIIM_CUDA(cudaEventCreate(&ev1));
        const bool dev = (opt.memory == FIIM_MEM_DEVICE);
        auto nnz_of = [&](const int *rp) -> long {
            if (!dev) return rp[n];
            int z = 0;
            if (cudaMemcpy(&z, rp + n, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
            return z;
        };
        const long nA = nnz_of(Ai), nG = nnz_of(Gi), nH = nnz_of(Hi);
        if (nA < 0 || nG < 0 || nH < 0) return set_error(FIIM_ECUDA, "reading row offsets failed");
        const size_t vsz = bf16 ? sizeof(__nv_bfloat16) : sizeof(float);
        const int max_blocks = num_sms() * 32;
        size_t bytes = csr_bytes(n, nA) + Arena::need(sizeof(float) * std::max<long>(nA, 1));
        // G and H: index arrays + FP64 staging share (reused) + low-precision values
        bytes += csr_bytes(n, nG) + csr_bytes(n, nH);
        bytes += Arena::need(vsz * std::max<long>(nG, 1)) + Arena::need(vsz * std::max<long>(nH, 1));
        bytes += 3 * Arena::need(sizeof(double) * n) + 11 * Arena::need(sizeof(float) * n);
        bytes += 2 * Arena::need(sizeof(DState)) + Arena::need(sizeof(mx::RState)) +
                 Arena::need(sizeof(double) * 4 * max_blocks) + 4096;
        FIIM_TRY(arena.reserve(bytes));
        FIIM_TRY(carve_csr(arena, A, n, nA));
        FIIM_TRY(carve_csr(arena, G, n, nG));   // G.v / H.v: FP64 staging, dropped after conversion
        FIIM_TRY(carve_csr(arena, H, n, nH));
        A32 = static_cast<float *>(arena.take(sizeof(float) * std::max<long>(nA, 1)));
        if (bf16) {
            G16 = static_cast<__nv_bfloat16 *>(arena.take(vsz * std::max<long>(nG, 1)));
            H16 = static_cast<__nv_bfloat16 *>(arena.take(vsz * std::max<long>(nH, 1)));
        } else {
            G32 = static_cast<float *>(arena.take(vsz * std::max<long>(nG, 1)));
            H32 = static_cast<float *>(arena.take(vsz * std::max<long>(nH, 1)));
        }
        double **d64[] = {&x, &b, &r64};
        for (auto pp : d64)
            if (!(*pp = static_cast<double *>(arena.take(sizeof(double) * n)))) return set_error(FIIM_ENOMEM, "arena");
        float **f32[] = {&D32, &e, &r, &r0, &p, &v, &s, &t, &pc, &sc, &tm};
        for (auto pp : f32)
            if (!(*pp = static_cast<float *>(arena.take(sizeof(float) * n)))) return set_error(FIIM_ENOMEM, "arena");
        st = static_cast<DState *>(arena.take(sizeof(DState)));
        sto = static_cast<DState *>(arena.take(sizeof(DState)));
        rs = static_cast<mx::RState *>(arena.take(sizeof(mx::RState)));
        partials = static_cast<double *>(arena.take(sizeof(double) * 4 * max_blocks));
        d_count = static_cast<unsigned long long *>(arena.take(sizeof(unsigned long long)));
        if (!A32 || !st || !sto || !rs || !partials || !d_count || (bf16 ? (!G16 || !H16) : (!G32 || !H32)))
            return set_error(FIIM_ENOMEM, "arena exhausted");
        FIIM_CUDA(cudaHostAlloc(&hst, 2 * sizeof(DState) + 64 + sizeof(mx::RState), cudaHostAllocDefault));
        h_count = reinterpret_cast<unsigned long long *>(reinterpret_cast<char *>(hst) + 2 * sizeof(DState) + 32);
        hrs = reinterpret_cast<mx::RState *>(reinterpret_cast<char *>(hst) + 2 * sizeof(DState) + 64);
        FIIM_CUDA(cudaMemsetAsync(st, 0, sizeof(DState), stream));
        FIIM_CUDA(cudaMemsetAsync(sto, 0, sizeof(DState), stream));
        FIIM_CUDA(cudaMemsetAsync(rs, 0, sizeof(mx::RState), stream));

        FIIM_TRY(upload_csr(A, nA, n, Ai, Aj, Av, 0, dev, stream, d_count, h_count));
        FIIM_TRY(upload_csr(G, nG, n, Gi, Gj, Gv, 1, dev, stream, d_count, h_count));
        FIIM_TRY(upload_csr(H, nH, n, Hi, Hj, Hv, 2, dev, stream, d_count, h_count));
        auto conv = [&](const double *in, long cnt, float *o32, __nv_bfloat16 *o16) -> int {
            if (cnt <= 0) return FIIM_OK;
            if (o16) mx::k_to_bf16<<<sgrid(mx::k_to_bf16, cnt), kThreads, 0, stream>>>(cnt, in, o16);
            else mx::k_to_f32<<<sgrid(mx::k_to_f32, cnt), kThreads, 0, stream>>>(cnt, in, o32);
            FIIM_CUDA(cudaGetLastError());
            return FIIM_OK;
        };
        FIIM_TRY(conv(A.v, A.nnz, A32, nullptr));
        FIIM_TRY(conv(G.v, G.nnz, G32, G16));
        FIIM_TRY(conv(H.v, H.nnz, H32, H16));
        // D^-1 in FP32: stage through r64.
        FIIM_CUDA(cudaMemcpyAsync(r64, IDv, sizeof(double) * n, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                  stream));
        FIIM_TRY(conv(r64, n, D32, nullptr));
        FIIM_CUDA(cudaStreamSynchronize(stream));
        G.v = nullptr;   // the FP64 factor values are not used past set-up
        H.v = nullptr;
        if (opt.autotune) {
            FIIM_TRY(tune(A, A32));
            if (bf16) {
                FIIM_TRY(tune(G, G16));
                FIIM_TRY(tune(H, H16));
            } else {
                FIIM_TRY(tune(G, G32));
                FIIM_TRY(tune(H, H32));
            }
        } else {
            FIIM_TRY(set_tile(A, 2048, stream));
            FIIM_TRY(set_tile(G, 2048, stream));
            FIIM_TRY(set_tile(H, 2048, stream));
        }
        // Sliced-diagonal copies of the inner products' values where the matrices allow them
        // (A's FP64 residual product keeps the CSR streams).
        const int vb = bf16 ? 2 : 4;
        FIIM_TRY(build_dia_structure(A, stream, 4));
        FIIM_TRY(place_dia(A, A32, stream));
        FIIM_TRY(build_dia_structure(G, stream, vb));
        FIIM_TRY(place_dia(G, bf16 ? (const void *)G16 : (const void *)G32, stream));
        FIIM_TRY(build_dia_structure(H, stream, vb));
        FIIM_TRY(place_dia(H, bf16 ? (const void *)H16 : (const void *)H32, stream));
        return build_graph();
    }

    int solve(const double *b_in, double *x_io, double tol, int nmax, fiim_result *res) {
        FIIM_CUDA(cudaSetDevice(device));
        const bool dev = (opt.memory == FIIM_MEM_DEVICE);
        FIIM_CUDA(cudaEventRecord(ev0, stream));
        FIIM_CUDA(cudaMemcpyAsync(b, b_in, sizeof(double) * n, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                  stream));
        FIIM_CUDA(cudaMemcpyAsync(x, x_io, sizeof(double) * n, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                  stream));
        DState hi = {};
        hi.tol = opt.inner_tol;
        hi.eps = 1.11022302462516e-16;
        hi.nmax = std::min(opt.inner_nmax, std::max(nmax, 1));
        hi.info = -1;
        hi.maxmsteps = (opt.variant == FIIM_ACIFIM) ? std::min(std::max(n, 2000) / 50, 40)
                                                     : std::min(std::max(n, 500) / 50, 20);
        hi.alpha_guard = (opt.variant == FIIM_ACIFIM);
        DState *hso = hst + 1;
        int total_iters = 0, steps = 0, launches = 0, info = 3;
        double nb = 0.0, nr = 0.0;
        auto residual = [&]() -> int {
            FIIM_CUDA(spmv_64(A, stream, x, EpiResid{b, r64}, sto, partials));
            FIIM_CUDA(cudaMemcpyAsync(hso, sto, sizeof(DState), cudaMemcpyDeviceToHost, stream));
            FIIM_CUDA(cudaStreamSynchronize(stream));
            ++launches;
            nr = std::sqrt(hso->ts);
            nb = std::sqrt(hso->tt);
            return FIIM_OK;
        };
        // The inner loop: the graph's WHILE node, or (FIIM_GRAPH=host) the host relaunching
        // a one-iteration graph until the device reports done.
        auto run_inner = [&]() -> int {
            if (!host_loop) {
                FIIM_CUDA(cudaGraphLaunch(exec, stream));
                return FIIM_OK;
            }
            int launched = 0, chunk = 1;
            for (;;) {
                for (int q = 0; q < chunk; ++q) FIIM_CUDA(cudaGraphLaunch(exec, stream));
                launched += chunk;
                FIIM_CUDA(cudaMemcpyAsync(&hst->done, &st->done, sizeof(int), cudaMemcpyDeviceToHost, stream));
                FIIM_CUDA(cudaStreamSynchronize(stream));
                if (hst->done) return FIIM_OK;
                if (launched > hst->nmax + 2) return set_error(FIIM_ETIMEOUT, "inner solve did not finish");
                chunk = std::min(chunk * 2, 16);
            }
        };
        FIIM_TRY(residual());
        const double r_start = nr;
        // Reliable updates: one inner solve over the whole iteration budget; its residual
        // replacements (refine_steps) move the correction into x and verify the stop in FP64.
        if (reliable) {
            if (nr <= tol * nb) {
                info = 0;
            } else if (nmax > 0) {
                *hst = hi;
                hst->nmax = nmax;
                hst->tol = tol * nb / nr;
                *hrs = mx::RState{};
                hrs->sigma = nr;
                hrs->inv_sigma = 1.0 / nr;
                hrs->goal = tol * nb;
                hrs->delta = opt.reliable;
                hrs->true_r = nr;
                hrs->max_verify = opt.max_refine;
                FIIM_CUDA(cudaMemcpyAsync(st, hst, sizeof(DState), cudaMemcpyHostToDevice, stream));
                FIIM_CUDA(cudaMemcpyAsync(rs, hrs, sizeof(mx::RState), cudaMemcpyHostToDevice, stream));
                mx::k_inner_init<<<sgrid(mx::k_inner_init, n), kThreads, 0, stream>>>(n, r64, sto, r, r0, p, e, st,
                                                                                       partials);
                FIIM_CUDA(cudaGetLastError());
                FIIM_TRY(run_inner());
                mx::k_promote<<<sgrid(mx::k_promote, n), kThreads, 0, stream>>>(n, e, x, sto);
                FIIM_CUDA(cudaGetLastError());
                FIIM_CUDA(cudaMemcpyAsync(hst, st, sizeof(DState), cudaMemcpyDeviceToHost, stream));
                FIIM_CUDA(cudaMemcpyAsync(hrs, rs, sizeof(mx::RState), cudaMemcpyDeviceToHost, stream));
                FIIM_TRY(residual());
                if (hst->info == -5) return set_error(FIIM_ETIMEOUT, "device loop guard tripped");
                steps = hrs->replacements;
                total_iters = hst->iter + ((hst->info == 1 || hst->info == 2) ? 1 : 0);
                launches += 2 + hst->loops * 9 + hrs->replacements * 2;
                info = (nr <= tol * nb) ? 0 : ((hst->info >= 1 && hst->info <= 3) ? hst->info : 3);
            }
        }
        while (!reliable) {
            if (nr <= tol * nb) { info = 0; break; }
            if (steps >= opt.max_refine || total_iters >= nmax) { info = 3; break; }
            *hst = hi;
            hst->nmax = std::min(hi.nmax, nmax - total_iters);
            // Ask the inner solve for no more than the reduction still missing (with a margin
            // of 3x), and never for less than inner_tol: the last step of a refinement then
            // stops as soon as the FP64 target is within reach.
            const double missing = tol * nb / nr;
            hst->tol = std::max(opt.inner_tol, std::min(0.5, missing / 3.0));
            FIIM_CUDA(cudaMemcpyAsync(st, hst, sizeof(DState), cudaMemcpyHostToDevice, stream));
            mx::k_inner_init<<<sgrid(mx::k_inner_init, n), kThreads, 0, stream>>>(n, r64, sto, r, r0, p, e, st, partials);
            FIIM_CUDA(cudaGetLastError());
            FIIM_TRY(run_inner());
            mx::k_promote<<<sgrid(mx::k_promote, n), kThreads, 0, stream>>>(n, e, x, sto);
            FIIM_CUDA(cudaGetLastError());
            FIIM_CUDA(cudaMemcpyAsync(hst, st, sizeof(DState), cudaMemcpyDeviceToHost, stream));
            const double prev = nr;
            FIIM_TRY(residual());
            ++steps;
            // iterations run: the completed ones plus the one a test stopped (info 0, 1, 2)
            total_iters += hst->iter + ((hst->info >= 0 && hst->info <= 2) ? 1 : 0);
            launches += 2 + hst->loops * 9;
            if (hst->info == -5) return set_error(FIIM_ETIMEOUT, "device loop guard tripped");
            if (!(nr < prev)) { info = (hst->info == 1 || hst->info == 2) ? hst->info : 1; break; }
        }
        FIIM_CUDA(cudaMemcpyAsync(x_io, x, sizeof(double) * n, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                  stream));
        FIIM_CUDA(cudaEventRecord(ev1, stream));
        FIIM_CUDA(cudaStreamSynchronize(stream));
        float ms = 0.f;
        FIIM_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
        if (res) {
            res->resval = r_start > 0 ? nr / r_start : nr;
            res->true_relres = nb > 0 ? nr / nb : nr;
            res->iter = total_iters;
            res->info = info;
            res->refine_steps = steps;
            res->device_ms = ms;
            res->launches = launches;
        }
        if (opt.verbose)
            std::cout << "Mixed-precision refinement: " << steps << " steps, " << total_iters
                      << " inner iterations, ||b-Ax||/||b|| = " << (nb > 0 ? nr / nb : nr) << ", info " << info << "\n";
        return FIIM_OK;
    }

    void destroy() {
        if (device >= 0) cudaSetDevice(device);
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
        if (hst) cudaFreeHost(hst);
        exec = nullptr;
        graph = nullptr;
        ev0 = ev1 = nullptr;
        stream = nullptr;
        hst = nullptr;
        for (DevCsr *M : {&A, &G, &H}) release_dia(*M);
        arena.release();
    }
};

}  // namespace fiim

int fiim_is_mixed(fiim_solver_t h) {
    return h && reinterpret_cast<fiim::SolverBase *>(h)->kind == fiim::kKindMixed;
}

int fiim_mixed_create(fiim_solver_t *out, int n, const int *Ai, const int *Aj, const double *Av,
                      const int *Gi, const int *Gj, const double *Gv, const double *IDv,
                      const int *Hi, const int *Hj, const double *Hv, const fiim_options *opt) {
    auto *s = new fiim::MixedSolver;
    const int rc = s->create(n, Ai, Aj, Av, Gi, Gj, Gv, IDv, Hi, Hj, Hv, *opt);
    if (rc != FIIM_OK) {
        s->destroy();
        delete s;
        return rc;
    }
    *out = reinterpret_cast<fiim_solver_t>(s);
    return FIIM_OK;
}

int fiim_mixed_solve(fiim_solver_t h, const double *b, double *x, double tol, int NMAX,
                     fiim_result *res) {
    return reinterpret_cast<fiim::MixedSolver *>(h)->solve(b, x, tol, NMAX, res);
}

int64_t fiim_mixed_device_bytes(fiim_solver_t h) {
    const auto *s = reinterpret_cast<fiim::MixedSolver *>(h);
    return (int64_t)(s->arena.cap + s->A.dia_bytes + s->G.dia_bytes + s->H.dia_bytes);
}

int fiim_mixed_destroy(fiim_solver_t h) {
    auto *s = reinterpret_cast<fiim::MixedSolver *>(h);
    s->destroy();
    delete s;
    return FIIM_OK;
}
