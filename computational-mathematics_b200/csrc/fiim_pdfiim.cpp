// Host construction of PDFIIM factors: G (upper, unit diagonal), D^{-1} and H (lower,
// unit diagonal) with dynamic sparsity patterns, one independent task per row.
// Restates pdfiim() (PDFIIM/src/parPrec.cpp:95-588) for pattern 'B' (both triangles of
// A drive the pattern), with the same operation order so the factors match the
// reference's bit for bit when both use the textbook LU (see lu_factor below):
//   * the row pattern is an insertion-ordered set; level sets are expanded from the
//     newest member back to the oldest (parPrec.cpp:150-219, 370-407);
//   * each lfill step solves B g = -a_col and B^T h = -a_row on the pattern, with
//     B = A restricted to the pattern and a floor max(1e-4, ftol) on missing or zero
//     diagonals (parPrec.cpp:260-290);
//   * entries below ftol * (filter norm) are dropped (parPrec.cpp:293-345);
//   * the next level set is grown from the first `kept` pattern members in solve
//     order (parPrec.cpp:366-385), as the reference does;
//   * D^{-1}_i = 1 / (h_i^T A g_i) over the kept entries (parPrec.cpp:502-532).
// Built with -ffp-contract=off.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "fiim_b200.h"

namespace {

// Insertion-ordered set of column indices < n.
struct PatternSet {
    std::vector<int> pos;    // position in `list`, or -1
    std::vector<int> list;   // members in insertion order
    explicit PatternSet(int n) : pos(n, -1) {}
    void push(int j) {
        if (pos[j] < 0) {
            pos[j] = (int)list.size();
            list.push_back(j);
        }
    }
    bool has(int j) const { return pos[j] >= 0; }
    void pop_newest() {
        pos[list.back()] = -1;
        list.pop_back();
    }
    void clear() {
        for (int j : list) pos[j] = -1;
        list.clear();
    }
    int size() const { return (int)list.size(); }
};

// Row-major LU with partial pivoting (first entry of largest magnitude), P B = L U;
// Golub & Van Loan Alg. 3.4.1 without blocking. A zero pivot column is left as is.
void lu_factor(int m, double *a, int *piv) {
    for (int k = 0; k < m; ++k) {
        int p = k;
        double best = std::fabs(a[(long)k * m + k]);
        for (int i = k + 1; i < m; ++i) {
            const double v = std::fabs(a[(long)i * m + k]);
            if (v > best) { best = v; p = i; }
        }
        piv[k] = p;
        if (a[(long)p * m + k] == 0.0) continue;
        if (p != k)
            for (int j = 0; j < m; ++j) std::swap(a[(long)k * m + j], a[(long)p * m + j]);
        const double d = a[(long)k * m + k];
        for (int i = k + 1; i < m; ++i) {
            const double l = a[(long)i * m + k] / d;
            a[(long)i * m + k] = l;
            for (int j = k + 1; j < m; ++j) a[(long)i * m + j] -= l * a[(long)k * m + j];
        }
    }
}

// Solve B x = y in place from lu_factor's output.
void lu_solve(int m, const double *a, const int *piv, double *y) {
    for (int k = 0; k < m; ++k)
        if (piv[k] != k) std::swap(y[k], y[piv[k]]);
    for (int i = 0; i < m; ++i) {
        double s = y[i];
        for (int j = 0; j < i; ++j) s -= a[(long)i * m + j] * y[j];
        y[i] = s;
    }
    for (int i = m - 1; i >= 0; --i) {
        double s = y[i];
        for (int j = i + 1; j < m; ++j) s -= a[(long)i * m + j] * y[j];
        y[i] = s / a[(long)i * m + i];
    }
}

// Solve B^T x = y in place from lu_factor's output.
void lu_solve_t(int m, const double *a, const int *piv, double *y) {
    for (int i = 0; i < m; ++i) {
        double s = y[i];
        for (int j = 0; j < i; ++j) s -= a[(long)j * m + i] * y[j];
        y[i] = s / a[(long)i * m + i];
    }
    for (int i = m - 1; i >= 0; --i) {
        double s = y[i];
        for (int j = i + 1; j < m; ++j) s -= a[(long)j * m + i] * y[j];
        y[i] = s;
    }
    for (int k = m - 1; k >= 0; --k)
        if (piv[k] != k) std::swap(y[k], y[piv[k]]);
}

struct Csr {
    const int *rp, *ci;
    const double *v;
};

// Add the strictly-lower-than-i columns of row j of M to the set (columns ascend).
inline void push_row_below(PatternSet &set, const Csr &M, int j, int i) {
    for (int l = M.rp[j]; l < M.rp[j + 1]; ++l) {
        if (M.ci[l] < i) set.push(M.ci[l]);
        else break;
    }
}

struct RowOut {
    std::vector<int> gj, hj;
    std::vector<double> gv, hv;
    double d;
};

// Everything one row task needs, reused across rows by a thread.
struct Work {
    PatternSet set;
    std::vector<int> inds, piv;
    std::vector<double> B, g, h;
    explicit Work(int n) : set(n) {}
};

double filter_norm(char filttype, const std::vector<double> &x, int len) {
    double nrm = 1.0;
    if (filttype == '1') {
        for (int j = 0; j < len; ++j) nrm += std::fabs(x[j]);
        nrm /= (len + 1);
    } else if (filttype == '2') {
        for (int j = 0; j < len; ++j) nrm += x[j] * x[j];
        nrm = std::sqrt(nrm);
    } else {
        for (int j = 0; j < len; ++j) nrm = (nrm < std::fabs(x[j])) ? std::fabs(x[j]) : nrm;
    }
    return nrm;
}

void build_row(int i, const Csr &A, const Csr &At, int prefill, int lfill, int postfill,
               double ftol, int warpsize, char filttype, Work &w, RowOut &out) {
    PatternSet &set = w.set;
    const double floor_diag = std::max(1e-4, ftol);
    // Level 1: columns < i of row i of A^T and of A (parPrec.cpp:144-151).
    push_row_below(set, At, i, i);
    push_row_below(set, A, i, i);
    // Pre-fill levels (parPrec.cpp:154-177): newest member first.
    for (int k = 2; k <= prefill; ++k) {
        const int len = set.size();
        for (int q = len - 1; q >= 0; --q) {
            const int jind = set.list[q];
            push_row_below(set, At, jind, i);
            push_row_below(set, A, jind, i);
        }
    }
    int c = 0, c2 = 0, tlen = 0;
    double ng = 0.0, nh = 0.0;
    for (int k = 1; k <= lfill; ++k) {
        c = 0;
        c2 = 0;
        ng = 0.0;
        int len = set.size();
        tlen = len;
        if (len == 0) break;
        // Cap the pattern below warpsize members, dropping the newest (parPrec.cpp:233).
        if (warpsize != -1)
            for (int j = len; j >= warpsize; --j) set.pop_newest();
        len = set.size();
        tlen = len;
        w.inds.assign(set.list.begin(), set.list.end());
        w.B.assign((size_t)len * len, 0.0);
        w.g.assign(len, 0.0);
        w.h.assign(len, 0.0);
        for (int j = 0; j < len; ++j) {
            const int row = w.inds[j];
            w.B[(size_t)j * len + j] = floor_diag;
            for (int kk = A.rp[row]; kk < A.rp[row + 1] && A.ci[kk] < i; ++kk) {
                const int col = A.ci[kk];
                if (set.has(col)) w.B[(size_t)j * len + set.pos[col]] = A.v[kk];
            }
            if (w.B[(size_t)j * len + j] == 0.0) w.B[(size_t)j * len + j] = floor_diag;
        }
        for (int kk = At.rp[i]; kk < At.rp[i + 1]; ++kk)
            if (set.has(At.ci[kk]) && At.ci[kk] < i) w.g[set.pos[At.ci[kk]]] = -At.v[kk];
        for (int kk = A.rp[i]; kk < A.rp[i + 1]; ++kk)
            if (set.has(A.ci[kk]) && A.ci[kk] < i) w.h[set.pos[A.ci[kk]]] = -A.v[kk];
        w.piv.resize(len);
        lu_factor(len, w.B.data(), w.piv.data());
        lu_solve(len, w.B.data(), w.piv.data(), w.g.data());
        lu_solve_t(len, w.B.data(), w.piv.data(), w.h.data());
        set.clear();
        ng = filter_norm(filttype, w.g, len);
        nh = filter_norm(filttype, w.h, len);
        for (int j = 0; j < len; ++j)
            if (std::fabs(w.g[j]) >= ftol * ng) { set.push(w.inds[j]); ++c; }
        for (int j = 0; j < len; ++j)
            if (std::fabs(w.h[j]) >= ftol * nh) { set.push(w.inds[j]); ++c2; }
        if ((c == 0 && c2 == 0) || c2 == warpsize) break;
        // Next level set from the first |set| entries of the solved pattern (parPrec.cpp:366-385).
        const int kept = set.size();
        for (int j = 0; j < kept; ++j) {
            push_row_below(set, At, w.inds[j], i);
            push_row_below(set, A, w.inds[j], i);
        }
        for (int m = 2; m <= postfill; ++m) {
            const int len2 = set.size();
            for (int q = len2 - 1; q >= 0; --q) {
                const int jind = set.list[q];
                push_row_below(set, At, jind, i);
                push_row_below(set, A, jind, i);
            }
        }
        if (set.size() == kept) break;
    }
    // Kept entries, sorted by index, then the unit diagonal (parPrec.cpp:460-500).
    auto collect = [&](const std::vector<double> &x, double nrm, std::vector<int> &oj,
                       std::vector<double> &ov) {
        std::vector<std::pair<int, double>> e;
        for (int j = 0; j < tlen; ++j)
            if (std::fabs(x[j]) >= ftol * nrm) e.emplace_back(w.inds[j], x[j]);
        std::sort(e.begin(), e.end(), [](const auto &a, const auto &b) { return a.first < b.first; });
        oj.resize(e.size() + 1);
        ov.resize(e.size() + 1);
        for (size_t q = 0; q < e.size(); ++q) {
            oj[q] = e[q].first;
            ov[q] = e[q].second;
        }
        oj[e.size()] = i;
        ov[e.size()] = 1.0;
    };
    if (tlen > 0) {
        collect(w.g, ng, out.gj, out.gv);
        collect(w.h, nh, out.hj, out.hv);
    } else {
        out.gj.assign(1, i); out.gv.assign(1, 1.0);
        out.hj.assign(1, i); out.hv.assign(1, 1.0);
    }
    set.clear();
    // D^{-1}_i = 1 / sum_j h_j (A g)_j over the kept patterns (parPrec.cpp:502-532).
    double s = 0.0;
    for (size_t j = 0; j < out.hj.size(); ++j) {
        const int hr = out.hj[j];
        const double hv = out.hv[j];
        int kk = A.rp[hr];
        size_t cc = 0;
        while (kk < A.rp[hr + 1] && cc < out.gj.size()) {
            if (A.ci[kk] == out.gj[cc]) {
                s += hv * A.v[kk] * out.gv[cc];
                ++kk;
                ++cc;
            } else if (A.ci[kk] < out.gj[cc]) {
                ++kk;
            } else {
                ++cc;
            }
        }
    }
    out.d = 1.0 / s;
}

struct Built {
    int n = 0;
    std::vector<int> Gi, Gj, Hi, Hj;
    std::vector<double> Gv, Hv, D;
};
thread_local Built g_built;

int build_all(int n, const int *Ai, const int *Aj, const double *Av, int prefill, int lfill,
              int postfill, double ftol, int warpsize, char filttype, Built &out) {
    const long nnz = Ai[n];
    // A^T by counting sort (columns ascend within each row).
    std::vector<int> tp(n + 1, 0), tc(nnz);
    std::vector<double> tv(nnz);
    for (long k = 0; k < nnz; ++k) tp[Aj[k] + 1]++;
    for (int r = 0; r < n; ++r) tp[r + 1] += tp[r];
    {
        std::vector<int> pos(tp.begin(), tp.end() - 1);
        for (int r = 0; r < n; ++r)
            for (int k = Ai[r]; k < Ai[r + 1]; ++k) {
                const int q = pos[Aj[k]]++;
                tc[q] = r;
                tv[q] = Av[k];
            }
    }
    const Csr A{Ai, Aj, Av}, At{tp.data(), tc.data(), tv.data()};
    std::vector<RowOut> rows(n);
    rows[0].gj.assign(1, 0); rows[0].gv.assign(1, 1.0);
    rows[0].hj.assign(1, 0); rows[0].hv.assign(1, 1.0);
    rows[0].d = 1.0 / Av[0];   // first stored entry of row 0 (parPrec.cpp:132)
#pragma omp parallel
    {
        Work w(n);
#pragma omp for schedule(dynamic, 256)
        for (int i = 1; i < n; ++i)
            build_row(i, A, At, prefill, lfill, postfill, ftol, warpsize, filttype, w, rows[i]);
    }
    // G: column i holds rows gj (ascending, diagonal last); assemble row-wise CSR.
    out.n = n;
    out.Gi.assign(n + 1, 0);
    for (int i = 0; i < n; ++i)
        for (int r : rows[i].gj) out.Gi[r + 1]++;
    for (int i = 0; i < n; ++i) out.Gi[i + 1] += out.Gi[i];
    out.Gj.resize(out.Gi[n]);
    out.Gv.resize(out.Gi[n]);
    {
        std::vector<int> pos(out.Gi.begin(), out.Gi.end() - 1);
        for (int i = 0; i < n; ++i)
            for (size_t q = 0; q < rows[i].gj.size(); ++q) {
                const int at = pos[rows[i].gj[q]]++;
                out.Gj[at] = i;
                out.Gv[at] = rows[i].gv[q];
            }
    }
    out.Hi.assign(n + 1, 0);
    for (int i = 0; i < n; ++i) out.Hi[i + 1] = out.Hi[i] + (int)rows[i].hj.size();
    out.Hj.resize(out.Hi[n]);
    out.Hv.resize(out.Hi[n]);
    out.D.resize(n);
    for (int i = 0; i < n; ++i) {
        std::copy(rows[i].hj.begin(), rows[i].hj.end(), out.Hj.begin() + out.Hi[i]);
        std::copy(rows[i].hv.begin(), rows[i].hv.end(), out.Hv.begin() + out.Hi[i]);
        out.D[i] = rows[i].d;
    }
    return FIIM_OK;
}

}  // namespace

extern "C" int fiim_pdfiim_build(int n, const int *Ai, const int *Aj, const double *Av, int prefill,
                                 int lfill, int postfill, double ftol, int warpsize, char filttype,
                                 char patt, int *nnzG, int *nnzH, double *Gv, int *Gj, int *Gi,
                                 double *D, double *Hv, int *Hj, int *Hi) {
    if (!Gv) {
        if (n <= 0 || !Ai || !Aj || !Av || !nnzG || !nnzH) return FIIM_EARG;
        if (patt != 'B') return FIIM_EARG;   // only the two-sided pattern is served
        if (warpsize == 0 || warpsize < -1) return FIIM_EARG;
        g_built = Built();
        const int rc = build_all(n, Ai, Aj, Av, prefill, lfill, postfill, ftol, warpsize, filttype, g_built);
        if (rc != FIIM_OK) return rc;
        *nnzG = g_built.Gi[n];
        *nnzH = g_built.Hi[n];
        return FIIM_OK;
    }
    if (g_built.n != n || !Gj || !Gi || !D || !Hv || !Hj || !Hi) return FIIM_EARG;
    std::memcpy(Gi, g_built.Gi.data(), sizeof(int) * (n + 1));
    std::memcpy(Gj, g_built.Gj.data(), sizeof(int) * g_built.Gj.size());
    std::memcpy(Gv, g_built.Gv.data(), sizeof(double) * g_built.Gv.size());
    std::memcpy(Hi, g_built.Hi.data(), sizeof(int) * (n + 1));
    std::memcpy(Hj, g_built.Hj.data(), sizeof(int) * g_built.Hj.size());
    std::memcpy(Hv, g_built.Hv.data(), sizeof(double) * g_built.Hv.size());
    std::memcpy(D, g_built.D.data(), sizeof(double) * n);
    g_built = Built();
    return FIIM_OK;
}
