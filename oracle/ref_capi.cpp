// ORACLE TEST INFRASTRUCTURE — not product code.
//
// extern "C" wrappers that let the test suite and bench.py's CPU-baseline leg call
// the reference's own, unmodified solve and construction code. This file is
// compiled together with the reference sources (read in place, never copied) and
// the MKL shim, once per package, by oracle/Makefile:
//   -DREF_AFIIM  : afiim (AFIIM/src/prec.hpp:99-114) + EPBiCGSTAB (AFIIM/src/bicgstab.hpp:82-100)
//   -DREF_PDFIIM : pdfiim (PDFIIM/src/parPrec.hpp:86-96) + EPBiCGSTAB (PDFIIM/src/bicgstab.hpp:75-86)
//   -DREF_ACIFIM : acifim (ACIFIM/src/prec.hpp:126-151) + PBiCGSTAB (ACIFIM/src/bicgstab.hpp:94-120)
// Each package becomes its own shared object (oracle/_ref/libref_<pkg>.so).

#include <chrono>
#include <cstring>
#include <cstdlib>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#if defined(REF_AFIIM)
#include "bicgstab.hpp"
#include "prec.hpp"
#include "rw_matrix.hpp"
#elif defined(REF_ACIFIM)
#include "bicgstab.hpp"
#include "prec.hpp"
#include "rw_matrix.hpp"
#elif defined(REF_PDFIIM)
#include "sparseMatrix.hpp"
#include "bicgstab.hpp"
#include "parPrec.hpp"
#include "rw_matrix.hpp"
#else
#error "define one of REF_AFIIM, REF_PDFIIM, REF_ACIFIM"
#endif

namespace {
// Owned copy of one factor set, handed to Python as an opaque pointer.
struct FactorSet {
    int n = 0;
    std::vector<double> Gv, IDv, Hv, Lv, Uv;
    std::vector<int> Gj, Gi, Hj, Hi, Lj, Li, Uj, Ui;
};

template <class T>
std::vector<T> take(T *p, long count) {
    return p ? std::vector<T>(p, p + count) : std::vector<T>();
}

template <class T>
void put(const std::vector<T> &v, T *dst) {
    if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(T));
}
}  // namespace

extern "C" {

void ref_set_threads(int t) {
#ifdef _OPENMP
    if (t > 0) omp_set_num_threads(t);
#endif
    (void)t;
}

int ref_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// Sizes of a factor set: out[0..4] = n, nnz(G), nnz(H), nnz(L), nnz(U).
void ref_factors_sizes(void *h, long *out) {
    auto *f = static_cast<FactorSet *>(h);
    out[0] = f->n;
    out[1] = (long)f->Gv.size();
    out[2] = (long)f->Hv.size();
    out[3] = (long)f->Lv.size();
    out[4] = (long)f->Uv.size();
}

// Copy a factor set into caller arrays (any pointer may be NULL to skip).
void ref_factors_get(void *h, double *Gv, int *Gj, int *Gi, double *IDv, double *Hv, int *Hj,
                     int *Hi, double *Lv, int *Lj, int *Li, double *Uv, int *Uj, int *Ui) {
    auto *f = static_cast<FactorSet *>(h);
    put(f->Gv, Gv); put(f->Gj, Gj); put(f->Gi, Gi); put(f->IDv, IDv);
    put(f->Hv, Hv); put(f->Hj, Hj); put(f->Hi, Hi);
    put(f->Lv, Lv); put(f->Lj, Lj); put(f->Li, Li);
    put(f->Uv, Uv); put(f->Uj, Uj); put(f->Ui, Ui);
}

void ref_factors_free(void *h) { delete static_cast<FactorSet *>(h); }

#if defined(REF_AFIIM) || defined(REF_ACIFIM)
// Matrix Market reader of the package (AFIIM/src/rw_matrix.cpp:62-216): 0-based CSR,
// columns sorted, symmetric input expanded. Returns a buffer the caller frees with
// ref_free_csr after copying.
struct CsrBuf { int n; double *Av; int *Aj; int *Ai; };
void *ref_read_matrix(const char *path, int *n, int *nnz) {
    auto *c = new CsrBuf{};
    read_coeff_matrix(path, &c->n, &c->Av, &c->Aj, &c->Ai);
    *n = c->n;
    *nnz = c->Ai[c->n];
    return c;
}
void ref_csr_get(void *h, double *Av, int *Aj, int *Ai) {
    auto *c = static_cast<CsrBuf *>(h);
    std::memcpy(Av, c->Av, sizeof(double) * c->Ai[c->n]);
    std::memcpy(Aj, c->Aj, sizeof(int) * c->Ai[c->n]);
    std::memcpy(Ai, c->Ai, sizeof(int) * (c->n + 1));
}
void ref_free_csr(void *h) {
    auto *c = static_cast<CsrBuf *>(h);
    delete[] c->Av; delete[] c->Aj; delete[] c->Ai;
    delete c;
}
// Dense right-hand side reader (AFIIM/src/rw_matrix.cpp:246-309).
int ref_read_rhs(const char *path, double *out, int cap) {
    int m = 0;
    double *B = nullptr;
    read_rhs_vector(path, &m, &B);
    if (m <= cap) std::memcpy(out, B, sizeof(double) * m);
    delete[] B;
    return m;
}
#endif

#if defined(REF_AFIIM)
void *ref_afiim_build(int n, double *Av, int *Aj, int *Ai, double dtol, int elemPerRowCol,
                      int growth, double eta, double shift) {
    double *Gv = nullptr, *Hv = nullptr, *IDv = nullptr;
    int *Gj = nullptr, *Gi = nullptr, *Hj = nullptr, *Hi = nullptr;
    afiim(n, Av, Aj, Ai, &Gv, &Gj, &Gi, &IDv, &Hv, &Hj, &Hi, dtol, elemPerRowCol, growth, eta,
          shift);
    auto *f = new FactorSet;
    f->n = n;
    f->Gi = take(Gi, n + 1); f->Gj = take(Gj, Gi[n]); f->Gv = take(Gv, Gi[n]);
    f->Hi = take(Hi, n + 1); f->Hj = take(Hj, Hi[n]); f->Hv = take(Hv, Hi[n]);
    f->IDv = take(IDv, n);
    delete[] Gv; delete[] Gj; delete[] Gi; delete[] Hv; delete[] Hj; delete[] Hi; delete[] IDv;
    return f;
}

void ref_afiim_solve(int n, double *Av, int *Aj, int *Ai, double *b, double tol, int NMAX,
                     double *Gv, int *Gj, int *Gi, double *IDv, double *Hv, int *Hj, int *Hi,
                     double *x, double *resval, int *iter, int verbose, int *info) {
    EPBiCGSTAB(n, Av, Aj, Ai, b, tol, NMAX, Gv, Gj, Gi, IDv, Hv, Hj, Hi, x, resval, iter, verbose,
               info);
}
#endif

#if defined(REF_ACIFIM)
// Returns the construction's own status (1 on a NaN pivot, ACIFIM/src/prec.cpp:857-858)
// through *cerr; the factor set is NULL when construction failed.
void *ref_acifim_build(int n, double *Av, int *Aj, int *Ai, double dtol1, double dtol2,
                       int elemPerRowCol, int growth, double eta, double shift, double coeff,
                       int element_limit, int filtit, int *cerr) {
    double *Gv = nullptr, *Hv = nullptr, *IDv = nullptr, *Lv = nullptr, *Uv = nullptr;
    int *Gj = nullptr, *Gi = nullptr, *Hj = nullptr, *Hi = nullptr;
    int *Lj = nullptr, *Li = nullptr, *Uj = nullptr, *Ui = nullptr;
    *cerr = acifim(n, Av, Aj, Ai, &Gv, &Gj, &Gi, &IDv, &Hv, &Hj, &Hi, &Lv, &Lj, &Li, &Uv, &Uj,
                   &Ui, dtol1, dtol2, elemPerRowCol, growth, eta, shift, coeff, element_limit,
                   filtit);
    if (*cerr != 0) return nullptr;
    auto *f = new FactorSet;
    f->n = n;
    f->Gi = take(Gi, n + 1); f->Gj = take(Gj, Gi[n]); f->Gv = take(Gv, Gi[n]);
    f->Hi = take(Hi, n + 1); f->Hj = take(Hj, Hi[n]); f->Hv = take(Hv, Hi[n]);
    f->Li = take(Li, n + 1); f->Lj = take(Lj, Li[n]); f->Lv = take(Lv, Li[n]);
    f->Ui = take(Ui, n + 1); f->Uj = take(Uj, Ui[n]); f->Uv = take(Uv, Ui[n]);
    f->IDv = take(IDv, n);
    delete[] Gv; delete[] Gj; delete[] Gi; delete[] Hv; delete[] Hj; delete[] Hi; delete[] IDv;
    delete[] Lv; delete[] Lj; delete[] Li; delete[] Uv; delete[] Uj; delete[] Ui;
    return f;
}

void ref_acifim_solve(int n, double *Av, int *Aj, int *Ai, double *b, double tol, int NMAX,
                      double *Gv, int *Gj, int *Gi, double *IDv, double *Hv, int *Hj, int *Hi,
                      double *Lv, int *Lj, int *Li, double *Uv, int *Uj, int *Ui, int nr,
                      char mode, double *x, double *resval, int *iter, int verbose, int *info) {
    PBiCGSTAB(n, Av, Aj, Ai, b, tol, NMAX, Gv, Gj, Gi, IDv, Hv, Hj, Hi, Lv, Lj, Li, Uv, Uj, Ui,
              nr, mode, x, resval, iter, verbose, info);
}
#endif

#if defined(REF_PDFIIM)
static void to_sparse(int n, int nnz, const double *v, const int *j, const int *i, int mtype,
                      sparseMatrix<int, int, double> &M) {
    M.resize(CSR, mtype, n, n, nnz);
    std::memcpy(M.v.data(), v, sizeof(double) * nnz);
    std::memcpy(M.j.data(), j, sizeof(int) * nnz);
    std::memcpy(M.i.data(), i, sizeof(int) * (n + 1));
}

void *ref_pdfiim_build(int n, double *Av, int *Aj, int *Ai, int prefill, int lfill,
                       int postfill, double ftol, int warpsize, char filttype, char patt) {
    sparseMatrix<int, int, double> A, G, H;
    std::vector<double> D;
    to_sparse(n, Ai[n], Av, Aj, Ai, GENERAL, A);
    pdfiim(A, G, D, H, prefill, lfill, postfill, ftol, warpsize, filttype, patt);
    auto *f = new FactorSet;
    f->n = n;
    f->Gi = G.i; f->Gj = G.j; f->Gv = G.v;
    f->Hi = H.i; f->Hj = H.j; f->Hv = H.v;
    f->IDv = D;
    return f;
}

// issym != 0: A holds only its upper triangle and is flagged SYMMETRIC, and the
// solver applies G^T in place of H (PDFIIM/src/bicgstab.cpp:145-153,189-192).
void ref_pdfiim_solve(int n, int issym, double *Av, int *Aj, int *Ai, double *b, double tol,
                      int NMAX, double *Gv, int *Gj, int *Gi, double *IDv, double *Hv, int *Hj,
                      int *Hi, double *x, double *resval, int *iter, int verbose, int *info) {
    sparseMatrix<int, int, double> A, G, H;
    to_sparse(n, Ai[n], Av, Aj, Ai, issym ? SYMMETRIC : GENERAL, A);
    to_sparse(n, Gi[n], Gv, Gj, Gi, UPPERTRI, G);
    if (!issym) to_sparse(n, Hi[n], Hv, Hj, Hi, LOWERTRI, H);
    std::vector<double> B(b, b + n), ID(IDv, IDv + n), X(x, x + n);
    EPBiCGSTAB(A, B, tol, NMAX, G, ID, H, X, resval, iter, verbose, info);
    std::memcpy(x, X.data(), sizeof(double) * n);
}

// A caller of the reference holds its system as sparseMatrix objects and std::vectors for
// as long as it solves. For timing the reference's call alone, the objects are built once
// here (ref_pdfiim_prepare) and each ref_pdfiim_run times EPBiCGSTAB by itself
// (PDFIIM/src/bicgstab.cpp:80-310): copying b and x in and out lies outside the clock.
struct PdfiimSystem {
    sparseMatrix<int, int, double> A, G, H;
    std::vector<double> B, ID, X;
};

void *ref_pdfiim_prepare(int n, int issym, double *Av, int *Aj, int *Ai, double *Gv, int *Gj,
                         int *Gi, double *IDv, double *Hv, int *Hj, int *Hi) {
    auto *s = new PdfiimSystem;
    to_sparse(n, Ai[n], Av, Aj, Ai, issym ? SYMMETRIC : GENERAL, s->A);
    to_sparse(n, Gi[n], Gv, Gj, Gi, UPPERTRI, s->G);
    if (!issym) to_sparse(n, Hi[n], Hv, Hj, Hi, LOWERTRI, s->H);
    s->ID.assign(IDv, IDv + n);
    s->B.assign(n, 0.0);
    s->X.assign(n, 0.0);
    return s;
}

// Returns the seconds spent inside EPBiCGSTAB (steady clock).
double ref_pdfiim_run(void *h, const double *b, double *x, double tol, int NMAX, double *resval,
                      int *iter, int *info) {
    auto *s = static_cast<PdfiimSystem *>(h);
    const size_t n = s->B.size();
    std::memcpy(s->B.data(), b, sizeof(double) * n);
    std::memcpy(s->X.data(), x, sizeof(double) * n);
    const auto t0 = std::chrono::steady_clock::now();
    EPBiCGSTAB(s->A, s->B, tol, NMAX, s->G, s->ID, s->H, s->X, resval, iter, 0, info);
    const auto t1 = std::chrono::steady_clock::now();
    std::memcpy(x, s->X.data(), sizeof(double) * n);
    return std::chrono::duration<double>(t1 - t0).count();
}

void ref_pdfiim_release(void *h) { delete static_cast<PdfiimSystem *>(h); }
#endif

}  // extern "C"
