// extern "C" entry points of include/fiim_b200.h and the C++ overloads with the
// reference's exact signatures (include/fiim_b200_compat.hpp), so that the reference's
// example drivers relink against this library unchanged.

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include <algorithm>

#include "fiim_b200.h"
#include "fiim_internal.h"
#include "fiim_solver.h"

namespace {

// Reference-facing calls reuse one solver per host thread while the problem shape is
// unchanged, so repeated solves skip allocation, tuning and graph capture. The device
// copies of the matrices and D^{-1} are also kept: each call stamps every input array
// (address, size, 64-bit content hash) and uploads the arrays again only if a stamp
// differs, so repeated solves with the same system upload only b and x0. The hash is
// recomputed on every call, so arrays changed in place are seen. fiim_dropin_cache(0),
// or FIIM_DROPIN_CACHE=0, uploads everything on every call instead.
struct Stamp {
    const void *p;
    size_t bytes;
    uint64_t h;
    bool operator==(const Stamp &o) const { return p == o.p && bytes == o.bytes && h == o.h; }
};

// The splitmix64 finalizer (Steele, Lea and Flood, "Fast splittable pseudorandom number
// generators", OOPSLA 2014), used as a mixing function.
inline uint64_t mix64(uint64_t z) {
    z ^= z >> 30;
    z *= 0xbf58476d1ce4e5b9ULL;
    z ^= z >> 27;
    z *= 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

// Sum over 8-byte words of mix(word ^ position key): a change of any word, or a swap of
// two, changes the sum by a pseudo-random 64-bit amount. Summed in parallel.
uint64_t content_hash(const void *p, size_t bytes) {
    const unsigned char *c = static_cast<const unsigned char *>(p);
    const long nw = (long)(bytes / 8);
    uint64_t acc = 0;
#pragma omp parallel for reduction(+ : acc) schedule(static) if (nw > (1L << 16))
    for (long i = 0; i < nw; ++i) {
        uint64_t w;
        std::memcpy(&w, c + 8 * i, 8);
        acc += mix64(w ^ (0x9e3779b97f4a7c15ULL * (uint64_t)(i + 1)));
    }
    uint64_t tail = 0;
    std::memcpy(&tail, c + 8 * nw, bytes - 8 * (size_t)nw);
    return acc + mix64(tail ^ 0xd1b54a32d192ed03ULL) + mix64((uint64_t)bytes);
}

Stamp stamp(const void *p, size_t bytes) { return Stamp{p, bytes, p ? content_hash(p, bytes) : 0}; }

void stamp_csr(std::vector<Stamp> &out, int n, const int *rp, const int *ci, const double *v) {
    if (!rp) {
        out.push_back(Stamp{nullptr, 0, 0});
        return;
    }
    const size_t nnz = (size_t)std::max(rp[n], 0);
    out.push_back(stamp(rp, sizeof(int) * (n + 1)));
    out.push_back(stamp(ci, sizeof(int) * nnz));
    out.push_back(stamp(v, sizeof(double) * nnz));
}

thread_local int g_cache = [] {
    const char *e = std::getenv("FIIM_DROPIN_CACHE");
    return (e && e[0] == '0' && e[1] == 0) ? 0 : 1;
}();

struct OneShot {
    fiim::Solver *s = nullptr;
    std::vector<long> key;
    std::vector<Stamp> stamps;   // of the arrays now on the device (empty: unknown)
    ~OneShot() {
        if (s) {
            s->destroy();
            delete s;
        }
    }
};
thread_local OneShot g_one;

int oneshot(int variant, int issym, char mode, int nr, int n, const double *Av, const int *Aj,
            const int *Ai, const double *b, double tol, int NMAX, const double *Gv, const int *Gj,
            const int *Gi, const double *IDv, const double *Hv, const int *Hj, const int *Hi,
            const double *Lv, const int *Lj, const int *Li, const double *Uv, const int *Uj,
            const int *Ui, double *x, double *resval, int *iter, int verbose, int *info) {
    if (n <= 0 || !Ai || !Aj || !Av || !b || !x || !Gi || !Gj || !Gv || !IDv || !resval || !iter || !info)
        return fiim::set_error(FIIM_EARG, "null argument or n <= 0");
    fiim_options o;
    fiim_options_default(&o);
    o.variant = variant;
    o.issym = issym;
    o.mode = mode;
    o.nr = nr;
    o.verbose = verbose;
    o.memory = FIIM_MEM_HOST;
    const bool combined = (variant == FIIM_ACIFIM && mode == 'C' && nr > 1);
    std::vector<long> key = {variant, issym, (long)mode, combined ? nr : 1, n, Ai[n], Gi[n],
                             (!issym && Hi) ? Hi[n] : -1, (combined && Li) ? Li[n] : -1,
                             (combined && Ui) ? Ui[n] : -1};
    int rc = FIIM_OK;
    std::vector<Stamp> st;
    auto stamp_all = [&] {
        stamp_csr(st, n, Ai, Aj, Av);
        stamp_csr(st, n, Gi, Gj, Gv);
        stamp_csr(st, n, Hi, Hj, Hv);
        stamp_csr(st, n, combined ? Li : nullptr, Lj, Lv);
        stamp_csr(st, n, combined ? Ui : nullptr, Uj, Uv);
        st.push_back(stamp(IDv, sizeof(double) * n));
    };
    auto report = [&](const fiim_result &r) {
        *resval = r.resval;
        *iter = r.iter;
        if (r.info >= 0) *info = r.info;   // NMAX < 0: the reference leaves info untouched
    };
    if (g_cache && g_one.s && g_one.key == key && !g_one.stamps.empty()) {
        // The same shape as the previous call, whose arrays are on the device: start the
        // solve on those copies at once and stamp the arrays while it runs. x is copied back
        // only if every stamp still matches; otherwise the result is discarded and the call
        // uploads the arrays and solves again.
        g_one.s->opt.verbose = verbose;
        FIIM_TRY(g_one.s->solve_start(b, x, tol, NMAX));
        stamp_all();
        if (st == g_one.stamps) {
            fiim_result r{};
            FIIM_TRY(g_one.s->solve_finish(x, &r));
            report(r);
            return FIIM_OK;
        }
        FIIM_TRY(g_one.s->solve_finish(nullptr, nullptr));
    } else if (g_cache) {
        stamp_all();
    }
    if (g_one.s && g_one.key == key && !issym) {
        g_one.stamps.clear();
        g_one.s->opt.verbose = verbose;
        rc = g_one.s->stage_inputs(b, x);   // ahead of the matrix copies
        if (rc == FIIM_OK) rc = g_one.s->reload(Ai, Aj, Av, Gi, Gj, Gv, IDv, Hi, Hj, Hv, Li, Lj, Lv, Ui, Uj, Uv);
        if (rc == FIIM_OK) g_one.stamps = st;
        else g_one.s->inputs_staged = false;
    } else {
        g_one.stamps.clear();
        if (g_one.s) {
            g_one.s->destroy();
            delete g_one.s;
            g_one.s = nullptr;
        }
        auto *s = new fiim::Solver;
        rc = s->create(n, Ai, Aj, Av, Gi, Gj, Gv, IDv, Hi, Hj, Hv, Li, Lj, Lv, Ui, Uj, Uv, o);
        if (rc != FIIM_OK) {
            s->destroy();
            delete s;
            return rc;
        }
        g_one.s = s;
        g_one.key = key;
        g_one.stamps = st;
    }
    if (rc != FIIM_OK) return rc;
    fiim_result r{};
    rc = g_one.s->solve(b, x, tol, NMAX, &r);
    if (rc != FIIM_OK) return rc;
    report(r);
    return FIIM_OK;
}

void throw_on(int rc) {
    if (rc != FIIM_OK) throw std::runtime_error(std::string("fiim_b200: ") + fiim::last_error());
}

}  // namespace

extern "C" {

const char *fiim_last_error(void) { return fiim::last_error(); }

int fiim_dropin_cache(int enable) {
    const int prev = g_cache;
    g_cache = enable ? 1 : 0;
    if (!g_cache) g_one.stamps.clear();
    return prev;
}

void fiim_options_default(fiim_options *o) {
    if (!o) return;
    std::memset(o, 0, sizeof *o);
    o->variant = FIIM_AFIIM;
    o->precision = FIIM_FP64;
    o->memory = FIIM_MEM_HOST;
    o->mode = 'E';
    o->nr = 1;
    o->autotune = 0;
    o->inner_tol = 1e-5;
    o->inner_nmax = 1000;
    o->max_refine = 50;
    o->verified = 0;
    o->max_restarts = 4;
    o->reliable = 0.01;
}

int fiim_EPBiCGSTAB_afiim(int n, double *Av, int *Aj, int *Ai, double *b, double tol, int NMAX,
                          double *Gv, int *Gj, int *Gi, double *IDv, double *Hv, int *Hj, int *Hi,
                          double *x, double *resval, int *iter, int verbose, int *info) {
    if (!Hv || !Hj || !Hi) return fiim::set_error(FIIM_EARG, "H is required");
    return oneshot(FIIM_AFIIM, 0, 'E', 1, n, Av, Aj, Ai, b, tol, NMAX, Gv, Gj, Gi, IDv, Hv, Hj, Hi,
                   nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, x, resval, iter, verbose,
                   info);
}

int fiim_EPBiCGSTAB_pdfiim(int n, int issym, double *Av, int *Aj, int *Ai, double *b, double tol,
                           int NMAX, double *Gv, int *Gj, int *Gi, double *ID, double *Hv, int *Hj,
                           int *Hi, double *x, double *resval, int *iter, int verbose, int *info) {
    if (!issym && (!Hv || !Hj || !Hi)) return fiim::set_error(FIIM_EARG, "H is required unless issym");
    return oneshot(FIIM_PDFIIM, issym ? 1 : 0, 'E', 1, n, Av, Aj, Ai, b, tol, NMAX, Gv, Gj, Gi, ID,
                   Hv, Hj, Hi, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, x, resval, iter,
                   verbose, info);
}

int fiim_PBiCGSTAB_acifim(int n, double *Av, int *Aj, int *Ai, double *b, double tol, int NMAX,
                          double *Gv, int *Gj, int *Gi, double *IDv, double *Hv, int *Hj, int *Hi,
                          double *Lv, int *Lj, int *Li, double *Uv, int *Uj, int *Ui, int nr,
                          char mode, double *x, double *resval, int *iter, int verbose, int *info) {
    if (mode != 'E' && mode != 'C')
        return fiim::set_error(FIIM_EARG, "ACIFIM mode '%c' applies triangular solves, not the factored inverse", mode);
    if (!Hv || !Hj || !Hi) return fiim::set_error(FIIM_EARG, "H is required");
    return oneshot(FIIM_ACIFIM, 0, mode, nr, n, Av, Aj, Ai, b, tol, NMAX, Gv, Gj, Gi, IDv, Hv, Hj,
                   Hi, Lv, Lj, Li, Uv, Uj, Ui, x, resval, iter, verbose, info);
}

int fiim_solver_create(fiim_solver_t *out, int n, const int *Ai, const int *Aj, const double *Av,
                       const int *Gi, const int *Gj, const double *Gv, const double *IDv,
                       const int *Hi, const int *Hj, const double *Hv, const int *Li,
                       const int *Lj, const double *Lv, const int *Ui, const int *Uj,
                       const double *Uv, const fiim_options *opt) {
    if (!out) return fiim::set_error(FIIM_EARG, "out is NULL");
    *out = nullptr;
    fiim_options o;
    if (opt) o = *opt;
    else fiim_options_default(&o);
    if (o.precision != FIIM_FP64) {
        return fiim_mixed_create(out, n, Ai, Aj, Av, Gi, Gj, Gv, IDv, Hi, Hj, Hv, &o);
    }
    auto *s = new fiim::Solver;
    const int rc = s->create(n, Ai, Aj, Av, Gi, Gj, Gv, IDv, Hi, Hj, Hv, Li, Lj, Lv, Ui, Uj, Uv, o);
    if (rc != FIIM_OK) {
        s->destroy();
        delete s;
        return rc;
    }
    *out = reinterpret_cast<fiim_solver_t>(s);
    return FIIM_OK;
}

int fiim_solver_solve(fiim_solver_t h, const double *b, double *x, double tol, int NMAX,
                      fiim_result *res) {
    if (!h || !b || !x) return fiim::set_error(FIIM_EARG, "null argument");
    if (fiim_is_mixed(h)) return fiim_mixed_solve(h, b, x, tol, NMAX, res);
    return reinterpret_cast<fiim::Solver *>(h)->solve(b, x, tol, NMAX, res);
}

int64_t fiim_solver_device_bytes(fiim_solver_t h) {
    if (!h) return -1;
    if (fiim_is_mixed(h)) return fiim_mixed_device_bytes(h);
    return (int64_t) reinterpret_cast<fiim::Solver *>(h)->device_bytes();
}

int fiim_solver_spmv_shape(fiim_solver_t h, int which, int *tile, int *form) {
    if (!h || !tile || !form || fiim_is_mixed(h)) return fiim::set_error(FIIM_EARG, "bad handle");
    auto *s = reinterpret_cast<fiim::Solver *>(h);
    const fiim::DevCsr *m[] = {&s->A, &s->G, &s->H, &s->L, &s->U};
    if (which < 0 || which > 4) return fiim::set_error(FIIM_EARG, "which in 0..4 (A, G, H, L, U)");
    *tile = m[which]->tile;
    *form = m[which]->dia ? fiim::kFormDia : m[which]->form;
    return FIIM_OK;
}

int fiim_solver_apply(fiim_solver_t h, int op, const double *x, double *y) {
    if (!h || fiim_is_mixed(h) || !x || !y) return fiim::set_error(FIIM_EARG, "bad argument");
    return reinterpret_cast<fiim::Solver *>(h)->apply(op, x, y);
}

int fiim_solver_kernel_times(fiim_solver_t h, int reps, int max_kernels, double *ms, double *bytes,
                             char *names, int name_len) {
    if (!h || fiim_is_mixed(h) || !ms || !bytes || reps < 1) return fiim::set_error(FIIM_EARG, "bad argument");
    return reinterpret_cast<fiim::Solver *>(h)->kernel_times(reps, max_kernels, ms, bytes, names, name_len);
}

int fiim_solver_mode(fiim_solver_t h) {
    if (!h) return fiim::set_error(FIIM_EARG, "bad handle");
    if (fiim_is_mixed(h)) return 1;
    auto *s = reinterpret_cast<fiim::Solver *>(h);
    return s->clustered ? 3 : s->persistent ? 2 : (s->use_cond ? 0 : 1);
}

int fiim_solver_set_wait_limit(fiim_solver_t h, int polls) {
    if (!h || fiim_is_mixed(h) || polls < 1) return fiim::set_error(FIIM_EARG, "bad argument");
    reinterpret_cast<fiim::Solver *>(h)->wait_limit = polls;
    return FIIM_OK;
}

int fiim_solver_test_stall(fiim_solver_t h) {
    if (!h || fiim_is_mixed(h)) return fiim::set_error(FIIM_EARG, "bad handle");
    auto *s = reinterpret_cast<fiim::Solver *>(h);
    if (!s->persistent) return fiim::set_error(FIIM_EARG, "the solver does not run as one cooperative launch");
    s->stall_next = true;
    return FIIM_OK;
}

int fiim_solver_kernel_times_seq(fiim_solver_t h, int reps, int max_kernels, double *ms, double *bytes,
                                 char *names, int name_len, double *body_ms) {
    if (!h || fiim_is_mixed(h) || !ms || !bytes || reps < 1) return fiim::set_error(FIIM_EARG, "bad argument");
    return reinterpret_cast<fiim::Solver *>(h)->kernel_times(reps, max_kernels, ms, bytes, names, name_len, true,
                                                             body_ms);
}

double fiim_solver_iteration_bytes(fiim_solver_t h) {
    if (!h || fiim_is_mixed(h)) return -1.0;
    return reinterpret_cast<fiim::Solver *>(h)->iteration_bytes();
}

double fiim_solver_matrix_bytes(fiim_solver_t h, int which) {
    if (!h || fiim_is_mixed(h) || which < 0 || which > 4) return -1.0;
    auto *s = reinterpret_cast<fiim::Solver *>(h);
    const fiim::DevCsr *m[] = {&s->A, &s->G, &s->H, &s->L, &s->U};
    const fiim::DevCsr &M = *m[which];
    if (M.dia) return (double)M.dsh * M.dvbytes * (double)M.ndiag + 4.0 * M.drs * M.nsl;
    return (double)M.nnz * (8 + (M.narrow ? 2 : 4)) + 4.0 * (M.n + 1) + (M.narrow ? 4.0 * M.nblk : 0.0) +
           8.0 * (M.nblk + 1);
}

int fiim_solver_destroy(fiim_solver_t h) {
    if (!h) return FIIM_OK;
    if (fiim_is_mixed(h)) return fiim_mixed_destroy(h);
    auto *s = reinterpret_cast<fiim::Solver *>(h);
    s->destroy();
    delete s;
    return FIIM_OK;
}

int fiim_spmv(int n, const int *Ai, const int *Aj, const double *Av, const double *x, double *y,
              int vec, void *stream) {
    return fiim::spmv_api(n, Ai, Aj, Av, x, y, vec, static_cast<cudaStream_t>(stream));
}

int fiim_prec_apply(int n, const int *Gi, const int *Gj, const double *Gv, const double *IDv,
                    const int *Hi, const int *Hj, const double *Hv, const double *r, double *z,
                    double *tm, void *stream) {
    return fiim::prec_api(n, Gi, Gj, Gv, IDv, Hi, Hj, Hv, r, z, tm, static_cast<cudaStream_t>(stream));
}

}  // extern "C"

// ---------------------------------------------------------------------------------
// C++ overloads with the reference's signatures (mangled names match the reference's
// libafiim.so exports). They throw std::runtime_error on a GPU-side failure, which the
// reference's CPU code could not report.

// AFIIM/src/bicgstab.hpp:82-100
void EPBiCGSTAB(int n, double *Av, int *Aj, int *Ai, double *b, double tol, int NMAX, double *Gv,
                int *Gj, int *Gi, double *IDv, double *Hv, int *Hj, int *Hi, double *x,
                double *resval, int *iter, int verbose, int *info) {
    throw_on(fiim_EPBiCGSTAB_afiim(n, Av, Aj, Ai, b, tol, NMAX, Gv, Gj, Gi, IDv, Hv, Hj, Hi, x,
                                   resval, iter, verbose, info));
}

// ACIFIM/src/bicgstab.hpp:94-120
void PBiCGSTAB(int n, double *Av, int *Aj, int *Ai, double *b, double tol, int NMAX, double *Gv,
               int *Gj, int *Gi, double *IDv, double *Hv, int *Hj, int *Hi, double *Lv, int *Lj,
               int *Li, double *Uv, int *Uj, int *Ui, int nr, char mode, double *x, double *resval,
               int *iter, int verbose, int *info) {
    throw_on(fiim_PBiCGSTAB_acifim(n, Av, Aj, Ai, b, tol, NMAX, Gv, Gj, Gi, IDv, Hv, Hj, Hi, Lv, Lj,
                                   Li, Uv, Uj, Ui, nr, mode, x, resval, iter, verbose, info));
}

// PDFIIM/src/bicgstab.hpp:75-86 takes sparseMatrix<int,int,double>. This class has the
// member layout of PDFIIM/src/sparseMatrix.hpp:68-75 (an ABI that must match for the
// reference's callers to link), and the SYMMETRIC tag value of PDFIIM/src/constants.hpp.
template <typename P, typename R, typename S>
class sparseMatrix {
public:
    int stype;
    int mtype;
    std::vector<S> v;
    std::vector<R> i, j;
    P r, c, nnz;
};

void EPBiCGSTAB(sparseMatrix<int, int, double> &A, std::vector<double> &b, double tol, int NMAX,
                sparseMatrix<int, int, double> &G, std::vector<double> &ID,
                sparseMatrix<int, int, double> &H, std::vector<double> &x, double *resval,
                int *iter, int verbose, int *info) {
    constexpr int kSymmetricTag = 1;
    const int issym = (A.mtype == kSymmetricTag);
    const int n = A.r;
    if ((int)x.size() < n || (int)b.size() < n || (int)ID.size() < n)
        throw std::runtime_error("fiim_b200: vector sizes smaller than A.r");
    throw_on(fiim_EPBiCGSTAB_pdfiim(n, issym, A.v.data(), A.j.data(), A.i.data(), b.data(), tol,
                                    NMAX, G.v.data(), G.j.data(), G.i.data(), ID.data(),
                                    issym ? nullptr : H.v.data(), issym ? nullptr : H.j.data(),
                                    issym ? nullptr : H.i.data(), x.data(), resval, iter, verbose,
                                    info));
}
