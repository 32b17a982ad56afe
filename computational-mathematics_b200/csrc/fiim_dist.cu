// Row-partitioned FP64 BiCGSTAB: one system split into contiguous row blocks, one block per
// rank (one process per GPU), each rank running the iteration of fiim_solver.cu
// (AFIIM/src/bicgstab.cpp:151-297, with PDFIIM's and ACIFIM-'E''s control constants) on its
// own rows.
//
// Layout. A rank owns rows [lo, hi) of A, G and H. The columns a matrix's rows reference
// outside [lo, hi) form its halo. Each matrix's columns are renumbered monotonically into an
// extended vector [halo below lo | owned rows | halo above hi], so every row keeps its
// stored entry order and the CSR-stream SpMV sums it exactly as on one GPU: given the same
// input values, each rank's rows come out bit-identical to the single-GPU product. Vectors
// that feed a product (x, p, s -> A / H; tm -> G; pc, sc -> A) are kept in the extended
// layout of their matrix; the others hold the owned rows only.
//
// Exchange. Before each product the owned entries other ranks need are packed into a send
// list and moved to the peers' halo slots (NCCL send/recv, one group per vector). Every
// reduction of the iteration is first reduced over the rank's rows by the unchanged kernels,
// which export the totals into a small per-rank array instead of applying the scalar step;
// the ranks then gather those arrays (NCCL all-gather), and a one-thread kernel on every rank
// sums them in rank order and applies the scalar step of the single-GPU solve. Every rank
// therefore holds the same scalars and takes the same termination decision. Three gathers
// per iteration: alpha after A pc, omega after A sc, and the tests after the x/r update,
// which also carries ||pc||^2, ||r||^2 and ||x||^2 (they are only read by the tests).
//
// Emulation. fiim_dist_emulate runs R row blocks in one process on one GPU through the same
// per-rank kernels, steps and launch shapes, with device copies in place of NCCL. Its
// results are those of an R-GPU run on the same GPU model, bit for bit: every rank's partial
// sums are the same and the gathered sums are added in the same order.

#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include "fiim_b200.h"
#include "fiim_internal.h"
#include "fiim_kernels.cuh"

namespace fiim {
namespace dist {

constexpr int kLoc = 8;   // totals a rank exports per gather
// Slots of the exported totals: r0.r (x/r update), ||pc||^2 (G product), ||r||^2 and ||x||^2
// (s update), r0.v (A pc), t.s and t.t (A sc). The start and the true residual use 0..1.
constexpr int kSlotR0r = 0, kSlotPc2 = 1, kSlotR2 = 2, kSlotAlpha = 4, kSlotOmega = 5;

enum Lay { LA = 0, LG = 1, LH = 2, NL = 3 };
enum Vec { VX = 0, VP, VS, VTM, VPC, VSC, NV };
constexpr int kLayOf[NV] = {LA, LH, LH, LG, LA, LA};

// ---------------------------------------------------------------- device pieces
template <class E>
struct ToLoc : E {   // epilogue E, with its totals exported instead of applied
    double *loc;
    __device__ void finish(DState *, const double *t) const {
#pragma unroll
        for (int j = 0; j < E::NR; ++j) loc[j] = t[j];
    }
};

template <int NR>
struct FinLoc {
    double *loc;
    __device__ void finish(DState *, const double *t) const {
#pragma unroll
        for (int j = 0; j < NR; ++j) loc[j] = t[j];
    }
};

struct FinCtl {   // the tests, with the norms the single-GPU kernels would have stored
    __device__ void finish(DState *st, const double *t) const {
        st->pc2 = t[kSlotPc2];
        st->r2 = t[kSlotR2];
        st->x2 = t[kSlotR2 + 1];
        FinControl{}.finish(st, t);
    }
};

// Sum the gathered totals in rank order and apply the scalar step.
template <int NR, class Fin>
static __global__ void k_gather_finish(const double *__restrict__ gath, int world, int slot, DState *st, Fin fin,
                                       int gated) {
    if (threadIdx.x != 0) return;
    if (gated && st->done) return;
    double t[NR];
#pragma unroll
    for (int j = 0; j < NR; ++j) {
        double s = gath[slot + j];
        for (int q = 1; q < world; ++q) s = __dadd_rn(s, gath[(size_t)q * kLoc + slot + j]);
        t[j] = s;
    }
    fin.finish(st, t);
}

// Send list of one vector: buf[k] = own[idx[k]].
static __global__ void __launch_bounds__(kThreads)
k_pack(const double *__restrict__ own, const int *__restrict__ idx, int cnt, double *__restrict__ buf,
       const DState *st, int gated) {
    pdl_enter();
    if (gated && st->done) return;
    for (int k = blockIdx.x * kThreads + threadIdx.x; k < cnt; k += gridDim.x * kThreads) buf[k] = own[idx[k]];
    pdl_release();
}

static CsrView<double> view(const DevCsr &M) { return CsrView<double>{M.rp, M.ci, M.v, (int)M.n}; }

// The single-GPU solver's deterministic shape: row blocks of at most 2047 entries, row form.
constexpr int kTile = 2048;
template <typename Epi>
static cudaError_t spmv(const DevCsr &M, cudaStream_t s, const double *x, const Epi &epi, DState *st,
                        double *partials) {
    if (M.narrow) {
        auto kern = k_spmv_rows<kTile, Epi, true>;
        return launch_k(kern, grid_for(kern, 1, M.nblk), 0, s, view(M), M.rb, M.eb, M.nblk, x, epi, st, partials,
                        NarrowCols{M.cd, M.cb});
    }
    auto kern = k_spmv_rows<kTile, Epi, false>;
    return launch_k(kern, grid_for(kern, 1, M.nblk), 0, s, view(M), M.rb, M.eb, M.nblk, x, epi, st, partials,
                    NarrowCols{});
}

// ---------------------------------------------------------------- host plan
// One matrix's rows on a rank: kept entries (MKL TRIANGULAR semantics for G and H, as the
// single-GPU upload: fill 1 keeps col >= row, fill 2 keeps col <= row), columns renumbered
// into the extended layout, and the halo.
struct Part {
    std::vector<int> rp, ci;
    std::vector<double> v;
};

struct Layout {
    int nb = 0, na = 0;
    std::vector<int> halo;        // global columns, ascending: nb below the owned rows, then na above
    std::vector<int> rcnt, roff;  // per peer: halo entries it owns, their offset in the extended vector
    std::vector<int> scnt, soff;  // per peer: owned entries it needs, their offset in the send list
    std::vector<int> sidx;        // owned (local) indices sent, peer by peer
    int *d_sidx = nullptr;
    int nsend() const { return (int)sidx.size(); }
};

static int owner_of(const int64_t *rs, int world, long c) {
    return (int)(std::upper_bound(rs, rs + world + 1, (int64_t)c) - rs) - 1;
}

// Builds the kept, renumbered rows and the halo of rows [rs[rank], rs[rank+1]) given with
// GLOBAL columns (rp local, 0-based at the block's first row). v may be NULL (structure only).
static int make_part(int rank, int world, const int64_t *rs, const int *rp, const int *ci, const double *v, int fill,
                     Part &out, Layout &L) {
    const long lo = rs[rank], hi = rs[rank + 1], n = rs[world];
    const int nloc = (int)(hi - lo);
    out.rp.assign(nloc + 1, 0);
    out.ci.clear();
    out.v.clear();
    std::vector<int> outside;
    for (int i = 0; i < nloc; ++i) {
        const long row = lo + i;
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            const int c = ci[k];
            if (c < 0 || c >= n) return set_error(FIIM_EARG, "row %ld has column %d outside [0, %ld)", row, c, n);
            if ((fill == 1 && c < row) || (fill == 2 && c > row)) continue;
            out.ci.push_back(c);
            if (v) out.v.push_back(v[k]);
            if (c < lo || c >= hi) outside.push_back(c);
        }
        out.rp[i + 1] = (int)out.ci.size();
    }
    std::sort(outside.begin(), outside.end());
    outside.erase(std::unique(outside.begin(), outside.end()), outside.end());
    L.halo.swap(outside);
    L.nb = (int)(std::lower_bound(L.halo.begin(), L.halo.end(), (int)lo) - L.halo.begin());
    L.na = (int)L.halo.size() - L.nb;
    const auto below_end = L.halo.begin() + L.nb;
    for (int &c : out.ci) {
        if (c < lo) c = (int)(std::lower_bound(L.halo.begin(), below_end, c) - L.halo.begin());
        else if (c < hi) c = L.nb + (int)(c - lo);
        else c = L.nb + nloc + (int)(std::lower_bound(below_end, L.halo.end(), c) - below_end);
    }
    // Halo entry k sits at k (below) or k + nloc (above) of the extended vector; the
    // entries of one owner are consecutive.
    L.rcnt.assign(world, 0);
    L.roff.assign(world, 0);
    for (size_t k = 0; k < L.halo.size(); ++k) {
        const int q = owner_of(rs, world, L.halo[k]);
        if (L.rcnt[q]++ == 0) L.roff[q] = (int)k < L.nb ? (int)k : (int)k + nloc;
    }
    return FIIM_OK;
}

// Halo entries of `L` owned by q, as global columns.
static const int *halo_of(const Layout &L, int q, int nloc) {
    const int off = L.roff[q];
    return L.halo.data() + (off < L.nb ? off : off - nloc);
}

// Send lists from the peers' needs (global columns), checked to be owned rows.
static int set_sends(Layout &L, long lo, long hi, const std::vector<std::vector<int>> &needs) {
    const int world = (int)needs.size();
    L.scnt.assign(world, 0);
    L.soff.assign(world, 0);
    L.sidx.clear();
    for (int q = 0; q < world; ++q) {
        L.soff[q] = (int)L.sidx.size();
        L.scnt[q] = (int)needs[q].size();
        for (int c : needs[q]) {
            if (c < lo || c >= hi) return set_error(FIIM_EARG, "peer %d asked for row %d outside [%ld, %ld)", q, c, lo, hi);
            L.sidx.push_back((int)(c - lo));
        }
    }
    return FIIM_OK;
}

// ---------------------------------------------------------------- one rank
enum KernelId { KINIT, K1, K2, K3, K4, K5, K6, K7, K8, K9, KRESID };
enum GatherId { GINIT, GALPHA, GOMEGA, GCTL, GRESID };

struct Rank {
    int rank = 0, world = 1, nloc = 0;
    long lo = 0, hi = 0, n = 0;
    fiim_options opt{};
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    Arena arena;
    DevCsr M[NL];
    Layout L[NL];
    double *IDv = nullptr, *b = nullptr, *r = nullptr, *r0 = nullptr, *v = nullptr, *t = nullptr;
    double *ext[NV] = {};
    double *sendbuf = nullptr, *loc = nullptr, *gath = nullptr, *partials = nullptr;
    DState *st = nullptr, *hst = nullptr;
    int *hflag = nullptr;   // pinned: done flags of the last two chunks
    int launches_body = 0, launches_start = 0, launches_resid = 0;

    double *own(int k) const { return ext[k] + L[kLayOf[k]].nb; }

    ~Rank() { release(); }
    void release() {
        if (hst) cudaFreeHost(hst);
        hst = nullptr;
        hflag = nullptr;
        arena.release();
        if (own_stream && stream) cudaStreamDestroy(stream);
        stream = nullptr;
    }

    // Device buffers and uploads; the parts and send lists are set.
    int setup(const Part (&P)[NL], const double *IDv_host) {
        const int max_blocks = num_sms() * 32;
        size_t bytes = 0;
        for (int l = 0; l < NL; ++l) bytes += csr_bytes(nloc, (long)P[l].ci.size()) + Arena::need(sizeof(int) * (L[l].nsend() + 1));
        long maxsend = 1;
        for (int l = 0; l < NL; ++l) maxsend = std::max<long>(maxsend, L[l].nsend());
        bytes += 6 * Arena::need(sizeof(double) * nloc);
        for (int k = 0; k < NV; ++k) bytes += Arena::need(sizeof(double) * (nloc + L[kLayOf[k]].halo.size()));
        bytes += Arena::need(sizeof(double) * maxsend) + Arena::need(sizeof(double) * kLoc) +
                 Arena::need(sizeof(double) * kLoc * world) + Arena::need(sizeof(double) * 4 * max_blocks) +
                 Arena::need(sizeof(DState)) + 1024;
        FIIM_TRY(arena.reserve(bytes));
        FIIM_CUDA(cudaMemsetAsync(arena.base, 0, bytes, stream));
        for (int l = 0; l < NL; ++l) {
            FIIM_TRY(carve_csr(arena, M[l], nloc, (long)P[l].ci.size()));
            L[l].d_sidx = static_cast<int *>(arena.take(sizeof(int) * (L[l].nsend() + 1)));
            if (!L[l].d_sidx) return set_error(FIIM_ENOMEM, "arena exhausted");
        }
        double **own_only[] = {&IDv, &b, &r, &r0, &v, &t};
        for (double **p : own_only)
            if (!(*p = static_cast<double *>(arena.take(sizeof(double) * nloc)))) return set_error(FIIM_ENOMEM, "arena exhausted");
        for (int k = 0; k < NV; ++k)
            if (!(ext[k] = static_cast<double *>(arena.take(sizeof(double) * (nloc + L[kLayOf[k]].halo.size())))))
                return set_error(FIIM_ENOMEM, "arena exhausted");
        sendbuf = static_cast<double *>(arena.take(sizeof(double) * maxsend));
        loc = static_cast<double *>(arena.take(sizeof(double) * kLoc));
        gath = static_cast<double *>(arena.take(sizeof(double) * kLoc * world));
        partials = static_cast<double *>(arena.take(sizeof(double) * 4 * max_blocks));
        st = static_cast<DState *>(arena.take(sizeof(DState)));
        if (!sendbuf || !loc || !gath || !partials || !st) return set_error(FIIM_ENOMEM, "arena exhausted");
        if (!hst) FIIM_CUDA(cudaHostAlloc(&hst, sizeof(DState) + 64, cudaHostAllocDefault));
        hflag = reinterpret_cast<int *>(reinterpret_cast<char *>(hst) + sizeof(DState) + 32);
        for (int l = 0; l < NL; ++l) {
            const Part &p = P[l];
            FIIM_TRY(upload_csr(M[l], (long)p.ci.size(), nloc, p.rp.data(), p.ci.data(), p.v.data(), 0, false, stream,
                                nullptr, nullptr));
            FIIM_TRY(set_tile(M[l], kTile, stream));
            if (L[l].nsend())
                FIIM_CUDA(cudaMemcpyAsync(L[l].d_sidx, L[l].sidx.data(), sizeof(int) * L[l].nsend(),
                                          cudaMemcpyHostToDevice, stream));
        }
        FIIM_CUDA(cudaMemcpyAsync(IDv, IDv_host, sizeof(double) * nloc, cudaMemcpyHostToDevice, stream));
        FIIM_CUDA(cudaStreamSynchronize(stream));
        // Launches of our kernels per step list (the packs of empty send lists are skipped).
        auto packs = [&](int k) { return L[kLayOf[k]].nsend() ? 1 : 0; };
        launches_start = packs(VX) + 2;
        launches_resid = packs(VX) + 2;
        launches_body = 9 + 3 + packs(VP) + 2 * packs(VTM) + packs(VPC) + packs(VS) + packs(VSC);
        return FIIM_OK;
    }

    int pack(int k, bool gated) {
        const Layout &Lk = L[kLayOf[k]];
        const int cnt = Lk.nsend();
        if (!cnt) return FIIM_OK;
        const int g = grid_for(k_pack, kThreads, cnt);
        FIIM_CUDA(launch_k(k_pack, g, 0, stream, (const double *)own(k), (const int *)Lk.d_sidx, cnt, sendbuf,
                           (const DState *)st, gated ? 1 : 0));
        return FIIM_OK;
    }

    int kernel(int id) {
        cudaStream_t s = stream;
        const long nn = nloc;
        const int gs = grid_for(k_update_s<FinLoc<2>>, kThreads, nn);
        const int gx = grid_for(k_update_xr<FinLoc<1>>, kThreads, nn);
        const int gp = grid_for(k_update_p, kThreads, nn);
        switch (id) {
            case KINIT:
                FIIM_CUDA(spmv(M[LA], s, ext[VX], ToLoc<EpiInit>{{b, own(VP), r0, r}, loc}, st, partials));
                break;
            case K1: FIIM_CUDA(spmv(M[LH], s, ext[VP], EpiScale{own(VTM), IDv}, st, partials)); break;
            case K2: FIIM_CUDA(spmv(M[LG], s, ext[VTM], ToLoc<EpiNorm>{{own(VPC)}, loc + kSlotPc2}, st, partials)); break;
            case K3: FIIM_CUDA(spmv(M[LA], s, ext[VPC], ToLoc<EpiAlpha>{{v, r0}, loc + kSlotAlpha}, st, partials)); break;
            case K4:
                FIIM_CUDA(launch_k(k_update_s<FinLoc<2>>, gs, 0, s, nn, (const double *)r, (const double *)v,
                                   (const double *)own(VX), own(VS), st, partials, FinLoc<2>{loc + kSlotR2}));
                break;
            case K5: FIIM_CUDA(spmv(M[LH], s, ext[VS], EpiScale{own(VTM), IDv}, st, partials)); break;
            case K6: FIIM_CUDA(spmv(M[LG], s, ext[VTM], EpiStore{own(VSC)}, st, partials)); break;
            case K7: FIIM_CUDA(spmv(M[LA], s, ext[VSC], ToLoc<EpiOmega>{{t, own(VS)}, loc + kSlotOmega}, st, partials)); break;
            case K8:
                FIIM_CUDA(launch_k(k_update_xr<FinLoc<1>>, gx, 0, s, nn, (const double *)own(VPC),
                                   (const double *)own(VSC), (const double *)own(VS), (const double *)t,
                                   (const double *)r0, own(VX), r, st, partials, FinLoc<1>{loc + kSlotR0r}));
                break;
            case K9:
                FIIM_CUDA(launch_k(k_update_p, gp, 0, s, nn, (const double *)r, (const double *)v, own(VP), st,
                                   cudaGraphConditionalHandle{}, 0));
                break;
            case KRESID:
                FIIM_CUDA(spmv(M[LA], s, ext[VX], ToLoc<EpiResid>{{b, nullptr}, loc}, st, partials));
                break;
            default: return set_error(FIIM_EARG, "unknown step");
        }
        return FIIM_OK;
    }

    int finish(int id) {
        cudaStream_t s = stream;
        switch (id) {
            case GINIT: k_gather_finish<1><<<1, 32, 0, s>>>(gath, world, 0, st, FinInit{}, 1); break;
            case GALPHA: k_gather_finish<1><<<1, 32, 0, s>>>(gath, world, kSlotAlpha, st, EpiAlpha{}, 1); break;
            case GOMEGA: k_gather_finish<2><<<1, 32, 0, s>>>(gath, world, kSlotOmega, st, EpiOmega{}, 1); break;
            case GCTL: k_gather_finish<4><<<1, 32, 0, s>>>(gath, world, kSlotR0r, st, FinCtl{}, 1); break;
            case GRESID: k_gather_finish<2><<<1, 32, 0, s>>>(gath, world, 0, st, EpiResid{}, 0); break;
            default: return set_error(FIIM_EARG, "unknown gather");
        }
        FIIM_CUDA(cudaGetLastError());
        return FIIM_OK;
    }

    void init_state(double tol, int nmax) {
        DState h = {};
        h.tol = tol;
        h.eps = 1.11022302462516e-16;                                    // AFIIM/src/bicgstab.cpp:108
        h.nmax = nmax;
        h.info = -1;
        const int ng = (int)n;
        if (opt.variant == FIIM_ACIFIM) h.maxmsteps = std::min(std::max(ng, 2000) / 50, 40);  // ACIFIM :132
        else h.maxmsteps = std::min(std::max(ng, 500) / 50, 20);                               // AFIIM :114
        h.alpha_guard = (opt.variant == FIIM_ACIFIM);
        *hst = h;
    }
};

// ---------------------------------------------------------------- transports
struct Transport {
    virtual ~Transport() {}
    virtual int exchange(int k) = 0;   // halo of vector k, after every rank packed it
    virtual int allgather() = 0;       // every rank's loc -> every rank's gath
};

// NCCL, loaded at run time: the library keeps no link-time dependency on it. A process that
// already holds libnccl (PyTorch loads its own) uses that copy; FIIM_NCCL_LIB names another.
struct NcclApi {
    decltype(&ncclGetUniqueId) getUniqueId = nullptr;
    decltype(&ncclCommInitRank) commInitRank = nullptr;
    decltype(&ncclCommDestroy) commDestroy = nullptr;
    decltype(&ncclAllGather) allGather = nullptr;
    decltype(&ncclSend) send = nullptr;
    decltype(&ncclRecv) recv = nullptr;
    decltype(&ncclGroupStart) groupStart = nullptr;
    decltype(&ncclGroupEnd) groupEnd = nullptr;
    decltype(&ncclGetErrorString) errorString = nullptr;
};

static const NcclApi *nccl_api() {
    static std::mutex mu;
    static NcclApi api;
    static int state = 0;
    std::lock_guard<std::mutex> lk(mu);
    if (state == 0) {
        const char *path = std::getenv("FIIM_NCCL_LIB");
        void *h = path ? dlopen(path, RTLD_NOW | RTLD_LOCAL) : dlopen("libnccl.so.2", RTLD_NOW | RTLD_NOLOAD);
        if (!h && !path) h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_LOCAL);
        state = -1;
        if (h) {
#define FIIM_NCCL_SYM(field, name) api.field = reinterpret_cast<decltype(api.field)>(dlsym(h, #name))
            FIIM_NCCL_SYM(getUniqueId, ncclGetUniqueId);
            FIIM_NCCL_SYM(commInitRank, ncclCommInitRank);
            FIIM_NCCL_SYM(commDestroy, ncclCommDestroy);
            FIIM_NCCL_SYM(allGather, ncclAllGather);
            FIIM_NCCL_SYM(send, ncclSend);
            FIIM_NCCL_SYM(recv, ncclRecv);
            FIIM_NCCL_SYM(groupStart, ncclGroupStart);
            FIIM_NCCL_SYM(groupEnd, ncclGroupEnd);
            FIIM_NCCL_SYM(errorString, ncclGetErrorString);
#undef FIIM_NCCL_SYM
            if (api.getUniqueId && api.commInitRank && api.commDestroy && api.allGather && api.send && api.recv &&
                api.groupStart && api.groupEnd && api.errorString)
                state = 1;
        }
    }
    return state == 1 ? &api : nullptr;
}

#define FIIM_NCCL(api, call)                                                                       \
    do {                                                                                           \
        ncclResult_t r_ = (call);                                                                  \
        if (r_ != ncclSuccess)                                                                     \
            return ::fiim::set_error(FIIM_ECUDA, "%s: %s", #call, (api)->errorString(r_));         \
    } while (0)

struct NcclTransport : Transport {
    Rank *R = nullptr;
    ncclComm_t comm = nullptr;
    const NcclApi *api = nullptr;
    int exchange(int k) override {
        const Layout &Lk = R->L[kLayOf[k]];
        bool any = false;
        for (int q = 0; q < R->world; ++q) any |= (Lk.scnt[q] > 0) || (Lk.rcnt[q] > 0);
        if (!any) return FIIM_OK;
        FIIM_NCCL(api, api->groupStart());
        for (int q = 0; q < R->world; ++q) {
            if (q == R->rank) continue;
            if (Lk.scnt[q])
                FIIM_NCCL(api, api->send(R->sendbuf + Lk.soff[q], Lk.scnt[q], ncclDouble, q, comm, R->stream));
            if (Lk.rcnt[q])
                FIIM_NCCL(api, api->recv(R->ext[k] + Lk.roff[q], Lk.rcnt[q], ncclDouble, q, comm, R->stream));
        }
        FIIM_NCCL(api, api->groupEnd());
        return FIIM_OK;
    }
    int allgather() override {
        FIIM_NCCL(api, api->allGather(R->loc, R->gath, kLoc, ncclDouble, comm, R->stream));
        return FIIM_OK;
    }
};

// All ranks in this process on one stream: device copies in place of NCCL.
struct LocalTransport : Transport {
    std::vector<Rank *> ranks;
    int exchange(int k) override {
        const int l = kLayOf[k];
        for (Rank *R : ranks) {
            const Layout &Lr = R->L[l];
            for (int q = 0; q < R->world; ++q) {
                if (q == R->rank || !Lr.rcnt[q]) continue;
                const Rank *Q = ranks[q];
                FIIM_CUDA(cudaMemcpyAsync(R->ext[k] + Lr.roff[q], Q->sendbuf + Q->L[l].soff[R->rank],
                                          sizeof(double) * Lr.rcnt[q], cudaMemcpyDeviceToDevice, R->stream));
            }
        }
        return FIIM_OK;
    }
    int allgather() override {
        for (Rank *R : ranks)
            for (int q = 0; q < R->world; ++q)
                FIIM_CUDA(cudaMemcpyAsync(R->gath + (size_t)q * kLoc, ranks[q]->loc, sizeof(double) * kLoc,
                                          cudaMemcpyDeviceToDevice, R->stream));
        return FIIM_OK;
    }
};

// ---------------------------------------------------------------- step lists
enum { SK, SX, SXU, SG };   // kernel, exchange (skipped once done), exchange (always), gather
struct Step {
    int kind, id;
};
static const Step kStart[] = {{SXU, VX}, {SK, KINIT}, {SG, GINIT}};
static const Step kBody[] = {{SX, VP},  {SK, K1}, {SX, VTM}, {SK, K2},     {SX, VPC}, {SK, K3},
                             {SG, GALPHA}, {SK, K4}, {SX, VS},  {SK, K5},     {SX, VTM}, {SK, K6},
                             {SX, VSC}, {SK, K7}, {SG, GOMEGA}, {SK, K8},     {SG, GCTL}, {SK, K9}};
static const Step kResid[] = {{SXU, VX}, {SK, KRESID}, {SG, GRESID}};

template <size_t N>
static int run(std::vector<Rank *> &ranks, const Step (&steps)[N], Transport &tr) {
    for (const Step &s : steps) {
        switch (s.kind) {
            case SK:
                for (Rank *R : ranks) FIIM_TRY(R->kernel(s.id));
                break;
            case SX:
            case SXU:
                for (Rank *R : ranks) FIIM_TRY(R->pack(s.id, s.kind == SX));
                FIIM_TRY(tr.exchange(s.id));
                break;
            case SG:
                FIIM_TRY(tr.allgather());
                for (Rank *R : ranks) FIIM_TRY(R->finish(s.id));
                break;
        }
    }
    return FIIM_OK;
}

// The iteration loop. Bodies are launched in chunks; the done flag of chunk j is read only
// after chunk j + 1 has been launched, and the loop stops after the first chunk whose
// predecessor's flag reads done. Every rank holds the same scalars, so every rank launches
// the same number of bodies (and NCCL operations) whatever its timing.
constexpr int kChunk = 4;
static int iterate(std::vector<Rank *> &ranks, Transport &tr, cudaGraphExec_t exec, int nmax, cudaEvent_t ev[2],
                   int *bodies) {
    Rank &R0 = *ranks[0];
    int launched = 0;
    for (int j = 0;; ++j) {
        for (int k = 0; k < kChunk; ++k) {
            if (exec) FIIM_CUDA(cudaGraphLaunch(exec, R0.stream));
            else FIIM_TRY(run(ranks, kBody, tr));
        }
        launched += kChunk;
        FIIM_CUDA(cudaMemcpyAsync(&R0.hflag[j & 1], &R0.st->done, sizeof(int), cudaMemcpyDeviceToHost, R0.stream));
        FIIM_CUDA(cudaEventRecord(ev[j & 1], R0.stream));
        if (j >= 1) {
            FIIM_CUDA(cudaEventSynchronize(ev[(j - 1) & 1]));
            if (R0.hflag[(j - 1) & 1]) break;
        }
        if (launched > std::max(nmax, 0) + 2 * kChunk + 2)
            return set_error(FIIM_ETIMEOUT, "solve not finished after %d iterations", launched);
    }
    *bodies = launched;
    return FIIM_OK;
}

static int check_options(const fiim_options &o) {
    if (o.variant < FIIM_AFIIM || o.variant > FIIM_ACIFIM) return set_error(FIIM_EARG, "bad variant");
    if (o.variant == FIIM_ACIFIM && o.mode != 'E')
        return set_error(FIIM_EARG, "the row-partitioned solve serves ACIFIM mode 'E' only");
    if (o.issym) return set_error(FIIM_EARG, "the row-partitioned solve takes the full A and H (expand first)");
    if (o.precision != FIIM_FP64) return set_error(FIIM_EARG, "the row-partitioned solve is FP64");
    return FIIM_OK;
}

static int check_starts(int world, const int64_t *rs) {
    if (world < 1 || !rs) return set_error(FIIM_EARG, "world >= 1 and row_starts are required");
    if (rs[0] != 0) return set_error(FIIM_EARG, "row_starts[0] must be 0");
    for (int q = 0; q < world; ++q)
        if (rs[q + 1] <= rs[q]) return set_error(FIIM_EARG, "rank %d owns no rows (row_starts must increase)", q);
    if (rs[world] > 0x7fffffffL) return set_error(FIIM_EARG, "n exceeds int32");
    return FIIM_OK;
}

// ---------------------------------------------------------------- multi-process handle
struct Dist {
    Rank R;
    NcclTransport tr;
    int *d_scratch = nullptr;   // status and plan exchange
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, evc[2] = {nullptr, nullptr};
    int device = -1;

    ~Dist() { destroy(); }

    // All ranks' statuses agree: the first failure, or FIIM_OK.
    int agree(int rc) {
        const int w = R.world;
        std::vector<int> all(w, 0);
        const int mine = rc;
        FIIM_CUDA(cudaMemcpyAsync(d_scratch, &mine, sizeof(int), cudaMemcpyHostToDevice, R.stream));
        FIIM_NCCL(tr.api, tr.api->allGather(d_scratch, d_scratch + 1, 1, ncclInt32, tr.comm, R.stream));
        FIIM_CUDA(cudaMemcpyAsync(all.data(), d_scratch + 1, sizeof(int) * w, cudaMemcpyDeviceToHost, R.stream));
        FIIM_CUDA(cudaStreamSynchronize(R.stream));
        for (int q = 0; q < w; ++q)
            if (all[q] != FIIM_OK) return q == R.rank ? all[q] : set_error(all[q], "rank %d failed during set-up", q);
        return FIIM_OK;
    }

    void destroy() {
        if (device >= 0) cudaSetDevice(device);
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        cudaEvent_t *evs[] = {&ev0, &ev1, &evc[0], &evc[1]};
        for (cudaEvent_t *e : evs)
            if (*e) cudaEventDestroy(*e), *e = nullptr;
        if (tr.comm && tr.api) tr.api->commDestroy(tr.comm);
        tr.comm = nullptr;
        if (d_scratch) cudaFree(d_scratch);
        d_scratch = nullptr;
        R.release();
    }
};

}  // namespace dist
}  // namespace fiim

using namespace fiim;
using namespace fiim::dist;

extern "C" int fiim_dist_unique_id(unsigned char *id) {
    if (!id) return set_error(FIIM_EARG, "id is required");
    const NcclApi *api = nccl_api();
    if (!api) return set_error(FIIM_ENODEV, "libnccl.so.2 could not be loaded (set FIIM_NCCL_LIB)");
    ncclUniqueId u;
    FIIM_NCCL(api, api->getUniqueId(&u));
    static_assert(sizeof(u) == FIIM_DIST_ID_BYTES, "ncclUniqueId size");
    std::memcpy(id, &u, sizeof(u));
    return FIIM_OK;
}

extern "C" int fiim_dist_partition(int n, const int *Ai, const int *Gi, const int *Hi, int world,
                                   int64_t *row_starts) {
    if (n <= 0 || !Ai || world < 1 || world > n || !row_starts) return set_error(FIIM_EARG, "bad arguments");
    // Balance the rank's streamed work: its rows' entries of A, G and H, plus one per row
    // for the vector passes.
    auto w = [&](int i) -> double {
        double s = 1.0 + (Ai[i + 1] - Ai[i]);
        if (Gi) s += Gi[i + 1] - Gi[i];
        if (Hi) s += Hi[i + 1] - Hi[i];
        return s;
    };
    double total = 0.0;
    for (int i = 0; i < n; ++i) total += w(i);
    row_starts[0] = 0;
    double acc = 0.0;
    int q = 1;
    for (int i = 0; i + 1 < n && q < world; ++i) {
        acc += w(i);
        // Block q - 1 ends after row i once it holds its share, or when every later rank
        // needs one of the remaining rows.
        if (acc >= total * q / world || n - (i + 1) == world - q) row_starts[q++] = i + 1;
    }
    row_starts[world] = n;
    return FIIM_OK;
}

extern "C" int fiim_dist_plan(int rank, int world, const int64_t *row_starts, const int *Mi, const int *Mj,
                              int fill, int *nbelow, int *nabove, int *nkept, int *halo, int *rp, int *cols) {
    FIIM_TRY(check_starts(world, row_starts));
    if (rank < 0 || rank >= world || !Mi || !Mj || !nbelow || !nabove || !nkept || fill < 0 || fill > 2)
        return set_error(FIIM_EARG, "bad arguments");
    Part P;
    Layout L;
    FIIM_TRY(make_part(rank, world, row_starts, Mi, Mj, nullptr, fill, P, L));
    *nbelow = L.nb;
    *nabove = L.na;
    *nkept = (int)P.ci.size();
    if (halo) std::copy(L.halo.begin(), L.halo.end(), halo);
    if (rp) std::copy(P.rp.begin(), P.rp.end(), rp);
    if (cols) std::copy(P.ci.begin(), P.ci.end(), cols);
    return FIIM_OK;
}

struct fiim_dist_s {
    fiim::dist::Dist d;
};

extern "C" int fiim_dist_create(fiim_dist_t *out, int rank, int world, const unsigned char *id, int device,
                                const int64_t *row_starts, const int *Ai, const int *Aj, const double *Av,
                                const int *Gi, const int *Gj, const double *Gv, const double *IDv,
                                const int *Hi, const int *Hj, const double *Hv, const fiim_options *opt) {
    if (!out || !id || world < 1 || rank < 0 || rank >= world) return set_error(FIIM_EARG, "bad rank, world or id");
    *out = nullptr;
    FIIM_TRY(check_device(nullptr));   // FIIM_ENODEV without a device
    const NcclApi *api = nccl_api();
    if (!api) return set_error(FIIM_ENODEV, "libnccl.so.2 could not be loaded (set FIIM_NCCL_LIB)");
    if (device >= 0) FIIM_CUDA(cudaSetDevice(device));
    int dev = 0;
    FIIM_TRY(check_device(&dev));
    std::unique_ptr<fiim_dist_s> h(new fiim_dist_s());
    Dist &D = h->d;
    Rank &R = D.R;
    D.device = dev;
    R.rank = rank;
    R.world = world;
    fiim_options_default(&R.opt);
    if (opt) R.opt = *opt;
    FIIM_CUDA(cudaStreamCreateWithFlags(&R.stream, cudaStreamNonBlocking));
    R.own_stream = true;
    D.tr.R = &R;
    D.tr.api = api;
    ncclUniqueId u;
    std::memcpy(&u, id, sizeof(u));
    FIIM_NCCL(api, api->commInitRank(&D.tr.comm, world, u, rank));
    if (cudaMalloc(&D.d_scratch, sizeof(int) * (1 + 2 * world)) != cudaSuccess) {
        cudaGetLastError();
        D.d_scratch = nullptr;
        return set_error(FIIM_ENOMEM, "device allocation failed");
    }
    // From here on every early return releases the communicator and buffers through the
    // handle's destructor.
    // Local checks and parts; every rank learns every status before the plan exchange.
    int rc = check_starts(world, row_starts);
    if (rc == FIIM_OK) rc = check_options(R.opt);
    if (rc == FIIM_OK && R.opt.memory != FIIM_MEM_HOST && R.opt.memory != FIIM_MEM_DEVICE) rc = set_error(FIIM_EARG, "bad memory");
    if (rc == FIIM_OK && (!Ai || !Aj || !Av || !Gi || !Gj || !Gv || !IDv || !Hi || !Hj || !Hv))
        rc = set_error(FIIM_EARG, "null array");
    Part P[NL];
    if (rc == FIIM_OK) {
        R.lo = row_starts[rank];
        R.hi = row_starts[rank + 1];
        R.n = row_starts[world];
        R.nloc = (int)(R.hi - R.lo);
        const int *rps[NL] = {Ai, Gi, Hi}, *cis[NL] = {Aj, Gj, Hj};
        const double *vs[NL] = {Av, Gv, Hv};
        const int fills[NL] = {0, 1, 2};
        for (int l = 0; l < NL && rc == FIIM_OK; ++l) rc = make_part(rank, world, row_starts, rps[l], cis[l], vs[l], fills[l], P[l], R.L[l]);
    }
    const int agreed = D.agree(rc);
    if (agreed != FIIM_OK) return agreed;
    // Plan exchange: every rank tells each owner which of its rows it needs, per matrix.
    for (int l = 0; l < NL; ++l) {
        Layout &Ll = R.L[l];
        std::vector<int> cnt(world), all((size_t)world * world);
        for (int q = 0; q < world; ++q) cnt[q] = Ll.rcnt[q];
        int *dc = nullptr;
        if (cudaMalloc(&dc, sizeof(int) * (world + (size_t)world * world)) != cudaSuccess) {
            cudaGetLastError();
            return set_error(FIIM_ENOMEM, "device allocation failed");
        }
        std::unique_ptr<int, decltype(&cudaFree)> dc_guard(dc, &cudaFree);
        FIIM_CUDA(cudaMemcpyAsync(dc, cnt.data(), sizeof(int) * world, cudaMemcpyHostToDevice, R.stream));
        FIIM_NCCL(api, api->allGather(dc, dc + world, world, ncclInt32, D.tr.comm, R.stream));
        FIIM_CUDA(cudaMemcpyAsync(all.data(), dc + world, sizeof(int) * world * world, cudaMemcpyDeviceToHost, R.stream));
        FIIM_CUDA(cudaStreamSynchronize(R.stream));
        std::vector<int> scnt(world);
        long ssum = 0, rsum = 0;
        for (int q = 0; q < world; ++q) {
            scnt[q] = all[(size_t)q * world + rank];
            ssum += scnt[q];
            rsum += Ll.rcnt[q];
        }
        int *dl = nullptr;
        if (cudaMalloc(&dl, sizeof(int) * (ssum + rsum + 1)) != cudaSuccess) {
            cudaGetLastError();
            return set_error(FIIM_ENOMEM, "device allocation failed");
        }
        std::unique_ptr<int, decltype(&cudaFree)> dl_guard(dl, &cudaFree);
        int *dneed = dl + ssum;   // my needs, by owner, in halo order
        std::vector<int> needs_flat;
        std::vector<int> noff(world, 0);
        for (int q = 0; q < world; ++q) {
            noff[q] = (int)needs_flat.size();
            const int *hq = halo_of(Ll, q, R.nloc);
            needs_flat.insert(needs_flat.end(), hq, hq + Ll.rcnt[q]);
        }
        if (rsum) FIIM_CUDA(cudaMemcpyAsync(dneed, needs_flat.data(), sizeof(int) * rsum, cudaMemcpyHostToDevice, R.stream));
        FIIM_NCCL(api, api->groupStart());
        long off = 0;
        for (int q = 0; q < world; ++q) {
            if (q == rank) continue;
            if (Ll.rcnt[q]) FIIM_NCCL(api, api->send(dneed + noff[q], Ll.rcnt[q], ncclInt32, q, D.tr.comm, R.stream));
            if (scnt[q]) FIIM_NCCL(api, api->recv(dl + off, scnt[q], ncclInt32, q, D.tr.comm, R.stream));
            off += scnt[q];
        }
        FIIM_NCCL(api, api->groupEnd());
        std::vector<int> got(ssum);
        if (ssum) FIIM_CUDA(cudaMemcpyAsync(got.data(), dl, sizeof(int) * ssum, cudaMemcpyDeviceToHost, R.stream));
        FIIM_CUDA(cudaStreamSynchronize(R.stream));
        std::vector<std::vector<int>> needs(world);
        off = 0;
        for (int q = 0; q < world; ++q) {
            if (q == rank) continue;
            needs[q].assign(got.begin() + off, got.begin() + off + scnt[q]);
            off += scnt[q];
        }
        // A bad request is recorded, not acted on: every rank keeps issuing the same NCCL
        // operations for every matrix, and the ranks agree on the status afterwards.
        const int src = set_sends(Ll, R.lo, R.hi, needs);
        if (rc == FIIM_OK) rc = src;
    }
    {
        const int a = D.agree(rc);
        if (a != FIIM_OK) return a;
    }
    rc = R.setup(P, IDv);
    {
        const int a = D.agree(rc);
        if (a != FIIM_OK) return a;
    }
    // One body with the state marked done resolves every launch shape; then the body is
    // captured as a graph with its NCCL operations (FIIM_DIST_GRAPH=0: direct launches).
    std::vector<Rank *> ranks{&R};
    {
        DState hs = {};
        hs.done = 1;
        *R.hst = hs;
        FIIM_CUDA(cudaMemcpyAsync(R.st, R.hst, sizeof(DState), cudaMemcpyHostToDevice, R.stream));
        FIIM_TRY(run(ranks, kBody, D.tr));
        FIIM_CUDA(cudaStreamSynchronize(R.stream));
    }
    const char *ge = std::getenv("FIIM_DIST_GRAPH");
    if (!(ge && ge[0] == '0')) {
        // Capture does not run anything, so ranks whose capture fails (and fall back to
        // direct launches) still issue the same NCCL operations as the others.
        if (cudaStreamBeginCapture(R.stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            const int crc = run(ranks, kBody, D.tr);
            cudaGraph_t g = nullptr;
            const cudaError_t ec = cudaStreamEndCapture(R.stream, &g);
            if (crc == FIIM_OK && ec == cudaSuccess && cudaGraphInstantiate(&D.exec, g, 0) == cudaSuccess) {
                D.graph = g;
            } else {
                if (g) cudaGraphDestroy(g);
                D.exec = nullptr;
            }
        }
        cudaGetLastError();
    }
    FIIM_CUDA(cudaEventCreate(&D.ev0));
    FIIM_CUDA(cudaEventCreate(&D.ev1));
    FIIM_CUDA(cudaEventCreateWithFlags(&D.evc[0], cudaEventDisableTiming));
    FIIM_CUDA(cudaEventCreateWithFlags(&D.evc[1], cudaEventDisableTiming));
    *out = h.release();
    return FIIM_OK;
}

// Solve on the given rows: shared by the NCCL handle (one rank) and the emulation (all ranks).
static int dist_solve(std::vector<Rank *> &ranks, Transport &tr, cudaGraphExec_t exec, const double *const *b,
                      double *const *x, bool dev_io, double tol, int nmax, cudaEvent_t ev0, cudaEvent_t ev1,
                      cudaEvent_t evc[2], fiim_result *res) {
    Rank &R0 = *ranks[0];
    cudaStream_t s = R0.stream;
    const cudaMemcpyKind in_kind = dev_io ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    const cudaMemcpyKind out_kind = dev_io ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    FIIM_CUDA(cudaEventRecord(ev0, s));
    for (size_t q = 0; q < ranks.size(); ++q) {
        Rank &R = *ranks[q];
        FIIM_CUDA(cudaMemcpyAsync(R.b, b[q], sizeof(double) * R.nloc, in_kind, s));
        FIIM_CUDA(cudaMemcpyAsync(R.own(VX), x[q], sizeof(double) * R.nloc, in_kind, s));
        R.init_state(tol, nmax);
        FIIM_CUDA(cudaMemcpyAsync(R.st, R.hst, sizeof(DState), cudaMemcpyHostToDevice, s));
    }
    FIIM_TRY(run(ranks, kStart, tr));
    int bodies = 0;
    FIIM_TRY(iterate(ranks, tr, exec, nmax, evc, &bodies));
    FIIM_TRY(run(ranks, kResid, tr));
    for (size_t q = 0; q < ranks.size(); ++q) {
        Rank &R = *ranks[q];
        FIIM_CUDA(cudaMemcpyAsync(R.hst, R.st, sizeof(DState), cudaMemcpyDeviceToHost, s));
        FIIM_CUDA(cudaMemcpyAsync(x[q], R.own(VX), sizeof(double) * R.nloc, out_kind, s));
    }
    FIIM_CUDA(cudaEventRecord(ev1, s));
    FIIM_CUDA(cudaStreamSynchronize(s));
    float ms = 0.f;
    FIIM_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
    const DState &h = *R0.hst;
    if (res) {
        res->resval = h.rc / h.ro;
        res->true_relres = std::sqrt(h.ts) / std::sqrt(h.tt);
        res->iter = h.iter;
        res->info = h.info;
        res->refine_steps = 0;
        res->device_ms = ms;
        res->launches = R0.launches_start + bodies * R0.launches_body + R0.launches_resid;
    }
    return FIIM_OK;
}

extern "C" int fiim_dist_solve(fiim_dist_t h, const double *b, double *x, double tol, int NMAX, fiim_result *res) {
    if (!h || !b || !x) return set_error(FIIM_EARG, "null argument");
    Dist &D = h->d;
    FIIM_CUDA(cudaSetDevice(D.device));
    std::vector<Rank *> ranks{&D.R};
    const double *bs[1] = {b};
    double *xs[1] = {x};
    return dist_solve(ranks, D.tr, D.exec, bs, xs, D.R.opt.memory == FIIM_MEM_DEVICE, tol, NMAX, D.ev0, D.ev1, D.evc,
                      res);
}

extern "C" int fiim_dist_destroy(fiim_dist_t h) {
    if (!h) return FIIM_OK;
    h->d.destroy();
    delete h;
    return FIIM_OK;
}

extern "C" int fiim_dist_emulate(int world, const int64_t *row_starts, int n, const int *Ai, const int *Aj,
                                 const double *Av, const int *Gi, const int *Gj, const double *Gv, const double *IDv,
                                 const int *Hi, const int *Hj, const double *Hv, const double *b, double *x,
                                 double tol, int NMAX, const fiim_options *opt, fiim_result *res) {
    FIIM_TRY(check_starts(world, row_starts));
    if (row_starts[world] != n) return set_error(FIIM_EARG, "row_starts[world] must be n");
    if (!Ai || !Aj || !Av || !Gi || !Gj || !Gv || !IDv || !Hi || !Hj || !Hv || !b || !x)
        return set_error(FIIM_EARG, "null array");
    fiim_options o;
    fiim_options_default(&o);
    if (opt) o = *opt;
    FIIM_TRY(check_options(o));
    if (o.memory != FIIM_MEM_HOST) return set_error(FIIM_EARG, "the emulation takes host arrays");
    FIIM_TRY(check_device(nullptr));
    std::vector<std::unique_ptr<Rank>> owned(world);
    std::vector<Rank *> ranks(world);
    cudaStream_t s = nullptr;
    FIIM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    } guard{s};
    std::vector<std::array<Part, NL>> parts(world);
    const int *rps[NL] = {Ai, Gi, Hi}, *cis[NL] = {Aj, Gj, Hj};
    const double *vs[NL] = {Av, Gv, Hv};
    const int fills[NL] = {0, 1, 2};
    for (int q = 0; q < world; ++q) {
        owned[q].reset(new Rank());
        Rank &R = *owned[q];
        ranks[q] = &R;
        R.rank = q;
        R.world = world;
        R.opt = o;
        R.stream = s;
        R.lo = row_starts[q];
        R.hi = row_starts[q + 1];
        R.n = n;
        R.nloc = (int)(R.hi - R.lo);
        for (int l = 0; l < NL; ++l) {
            // The block's rows with offsets from its first entry.
            const int base = rps[l][R.lo];
            std::vector<int> rp(R.nloc + 1);
            for (int i = 0; i <= R.nloc; ++i) rp[i] = rps[l][R.lo + i] - base;
            FIIM_TRY(make_part(q, world, row_starts, rp.data(), cis[l] + base, vs[l] + base, fills[l], parts[q][l],
                               R.L[l]));
        }
    }
    for (int l = 0; l < NL; ++l)
        for (int q = 0; q < world; ++q) {
            std::vector<std::vector<int>> needs(world);
            for (int p = 0; p < world; ++p) {
                if (p == q) continue;
                const Layout &Lp = ranks[p]->L[l];
                const int *hp = halo_of(Lp, q, ranks[p]->nloc);
                needs[p].assign(hp, hp + Lp.rcnt[q]);
            }
            FIIM_TRY(set_sends(ranks[q]->L[l], ranks[q]->lo, ranks[q]->hi, needs));
        }
    for (int q = 0; q < world; ++q) {
        Part P[NL];
        for (int l = 0; l < NL; ++l) P[l] = std::move(parts[q][l]);
        FIIM_TRY(ranks[q]->setup(P, IDv + ranks[q]->lo));
    }
    LocalTransport tr;
    tr.ranks = ranks;
    std::vector<const double *> bs(world);
    std::vector<double *> xs(world);
    for (int q = 0; q < world; ++q) {
        bs[q] = b + ranks[q]->lo;
        xs[q] = x + ranks[q]->lo;
    }
    cudaEvent_t ev0, ev1, evc[2];
    FIIM_CUDA(cudaEventCreate(&ev0));
    FIIM_CUDA(cudaEventCreate(&ev1));
    FIIM_CUDA(cudaEventCreateWithFlags(&evc[0], cudaEventDisableTiming));
    FIIM_CUDA(cudaEventCreateWithFlags(&evc[1], cudaEventDisableTiming));
    const int rc = dist_solve(ranks, tr, nullptr, bs.data(), xs.data(), false, tol, NMAX, ev0, ev1, evc, res);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    cudaEventDestroy(evc[0]);
    cudaEventDestroy(evc[1]);
    if (rc == FIIM_OK && res) res->launches *= world;
    return rc;
}
