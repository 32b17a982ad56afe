// The sequential sweep shared by the AFIIM and ACIFIM factor constructions on the host
// (AFIIM/src/prec.cpp:101-767, ACIFIM/src/prec.cpp:127-1052): a sparse accumulator walked in
// the reference's order, the split of A into diagonal, strictly lower rows and strictly upper
// columns, and the assembly of the factors' per-index lists into CSR.
#pragma once

#include <cmath>
#include <vector>

namespace fiim {
namespace sweep {

struct Entry {
    int idx;
    double v;
};
using List = std::vector<Entry>;

// Sparse accumulator over [0, n): dense values and a chain of touched indices, newest first.
struct Accum {
    std::vector<double> val;
    std::vector<int> link;   // -1: untouched; else the index touched before this one (-2: none)
    int head = -2, count = 0;
    explicit Accum(int n) : val(n, 0.0), link(n, -1) {}
    // First touch assigns (as the reference does), later touches add.
    void add(int k, double v) {
        if (link[k] == -1) {
            val[k] = v;
            link[k] = head;
            head = k;
            ++count;
        } else {
            val[k] += v;
        }
    }
    template <class F>
    void walk(F f) const {
        for (int q = 0, k = head; q < count; ++q, k = link[k]) f(k);
    }
    void clear() {
        for (int q = 0, k = head; q < count; ++q) {
            const int nx = link[k];
            link[k] = -1;
            val[k] = 0.0;
            k = nx;
        }
        head = -2;
        count = 0;
    }
};

struct Factors {
    int n = 0;
    std::vector<int> Gi, Gj, Hi, Hj, Li, Lj, Ui, Uj;
    std::vector<double> Gv, Hv, Lv, Uv, IDv;
};

// Rows of per-index lists as CSR, row i = lists[i] in order (G from G^T, U from U^T).
inline void rows_of(const std::vector<List> &lists, std::vector<int> &rp, std::vector<int> &ci, std::vector<double> &v) {
    const int n = (int)lists.size();
    rp.assign(n + 1, 0);
    for (int i = 0; i < n; ++i) rp[i + 1] = rp[i] + (int)lists[i].size();
    ci.resize(rp[n]);
    v.resize(rp[n]);
    for (int i = 0, at = 0; i < n; ++i)
        for (const Entry &e : lists[i]) {
            ci[at] = e.idx;
            v[at++] = e.v;
        }
}

// Transposed lists as CSR: lists[i] holds (row, value) entries of column i; a row's entries
// come out in ascending column order (H from H^T, L from L^T; prec.cpp:917-1003).
inline void rows_of_transposed(const std::vector<List> &lists, std::vector<int> &rp, std::vector<int> &ci,
                               std::vector<double> &v) {
    const int n = (int)lists.size();
    rp.assign(n + 1, 0);
    for (const List &l : lists)
        for (const Entry &e : l) rp[e.idx + 1]++;
    for (int i = 0; i < n; ++i) rp[i + 1] += rp[i];
    ci.resize(rp[n]);
    v.resize(rp[n]);
    std::vector<int> pos(rp.begin(), rp.end() - 1);
    for (int i = 0; i < n; ++i)
        for (const Entry &e : lists[i]) {
            ci[pos[e.idx]] = i;
            v[pos[e.idx]++] = e.v;
        }
}

// A split into its diagonal, strictly lower rows (CSR, row order) and strictly upper columns
// (CSC, rows ascending), as both constructions do first (ACIFIM/src/prec.cpp:279-344,
// AFIIM/src/prec.cpp:239-306). A zero or missing diagonal reads `dzero`.
struct Split {
    std::vector<double> d;
    std::vector<int> lp, lcol, up, urow;
    std::vector<double> lval, uval;
};

inline void split(int n, const int *Ai, const int *Aj, const double *Av, double dzero, Split &a) {
    a.d.assign(n, 0.0);
    a.lp.assign(n + 1, 0);
    a.up.assign(n + 1, 0);
    for (int i = 0; i < n; ++i)
        for (int q = Ai[i]; q < Ai[i + 1]; ++q) {
            if (Aj[q] > i) a.up[Aj[q] + 1]++;
            else if (Aj[q] < i) a.lp[i + 1]++;
        }
    for (int i = 0; i < n; ++i) {
        a.lp[i + 1] += a.lp[i];
        a.up[i + 1] += a.up[i];
    }
    a.lcol.resize(a.lp[n]);
    a.lval.resize(a.lp[n]);
    a.urow.resize(a.up[n]);
    a.uval.resize(a.up[n]);
    std::vector<int> upos(a.up.begin(), a.up.end() - 1);
    for (int i = 0, lq = 0; i < n; ++i) {
        for (int q = Ai[i]; q < Ai[i + 1]; ++q) {
            const int c = Aj[q];
            if (c > i) {
                a.urow[upos[c]] = i;
                a.uval[upos[c]++] = Av[q];
            } else if (c < i) {
                a.lcol[lq] = c;
                a.lval[lq++] = Av[q];
            } else {
                a.d[i] = Av[q];
            }
        }
        if (a.d[i] == 0.0) a.d[i] = dzero;
    }
}

}  // namespace sweep
}  // namespace fiim
