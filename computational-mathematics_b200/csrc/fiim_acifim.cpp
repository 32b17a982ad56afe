// ACIFIM factor construction on the host: the same G, D^{-1}, H (and L, U) as acifim
// (ACIFIM/src/prec.cpp:127-1052), bit for bit, for callers and benchmarks that need ACIFIM
// factors without the reference library.
//
// The method builds, for r = 1 .. n-1 in turn, column r of the upper unit factor G, row r of
// the lower unit factor H and the pivot 1/s_r of D^{-1}, from the strictly upper column r
// (b) and strictly lower row r (c) of A:
//   t_b = H b, t_c = c G            (sparse accumulators, then drop-filtered, stored in U, L)
//   g_r = -G D^{-1} t_b, h_r = -t_c D^{-1} H   (filtered relative to running column norms)
//   s_r = d_r + t_b^T D^{-1} t_c - c g_r - h_r b
// Every sum runs in the reference's order: an accumulator is walked newest index first
// (the order its linked list is traversed, prec.cpp:391-402), which fixes both the order of
// the stored entries and the order of the Schur complement's sum; products are evaluated
// left to right as written there, and this file is compiled without FMA contraction.
// growth and elemPerRowCol only size the reference's buffers and change nothing here.

#include <cmath>
#include <cstring>
#include <vector>

#include "fiim_b200.h"
#include "fiim_internal.h"
#include "fiim_sweep.h"

namespace {

using fiim::sweep::Accum;
using fiim::sweep::Entry;
using fiim::sweep::Factors;
using fiim::sweep::List;
using fiim::sweep::rows_of;
using fiim::sweep::rows_of_transposed;

// Drop filter of t_b or t_c (prec.cpp:383-414, 535-565): entries with
// |D^{-1}_k val_k| <= (m * tol) / norm_k are zeroed, first with m = 1; while more than
// `limit` survive, the pass repeats (m = 1, then coeff, coeff^2, ...), at most filtit more
// passes. Returns the survivors.
int drop(Accum &a, const std::vector<double> &idv, double tol, const std::vector<double> &norm, int limit,
         int filtit, double coeff) {
    auto pass = [&](double m) {
        int cut = 0;
        a.walk([&](int k) {
            if (std::fabs(idv[k] * a.val[k]) <= m * tol / norm[k]) {
                a.val[k] = 0.0;
                ++cut;
            }
        });
        return cut;
    };
    int cut = pass(1.0);
    double mult = 1.0;
    for (int l = 1; a.count - cut > limit && l <= filtit; ++l) {
        cut = pass(mult);
        mult *= coeff;
    }
    return a.count - cut;
}

int build(int n, const int *Ai, const int *Aj, const double *Av, double dtol1, double dtol2, double eta,
          double shift, double coeff, int limit, int filtit, Factors &out) {
    fiim::sweep::Split a;
    fiim::sweep::split(n, Ai, Aj, Av, dtol2, a);
    const std::vector<double> &d = a.d, &lval = a.lval, &uval = a.uval;
    const std::vector<int> &lp = a.lp, &lcol = a.lcol, &up = a.up, &urow = a.urow;

    std::vector<double> &idv = out.IDv;
    idv.assign(n, 0.0);
    {
        const double s = d[0] + shift * std::fabs(d[0]);
        idv[0] = (std::fabs(s) < eta) ? 1.0 / (1e-4 + dtol2) : 1.0 / s;
    }
    // Column r of G and row r of H as built (their diagonal last); G^T, H^T, U^T, L^T grow
    // by one entry per index per step.
    std::vector<List> gcol(n), hrow(n), gt(n), ht(n), ut(n), lt(n);
    gcol[0] = {{0, 1.0}};
    hrow[0] = {{0, 1.0}};
    gt[0] = {{0, 1.0}};
    ht[0] = {{0, 1.0}};
    for (int i = 0; i < n; ++i) {
        ut[i] = {{i, 1.0}};
        lt[i] = {{i, 1.0}};
    }
    std::vector<double> gn(n, 1.0), hn(n, 1.0), gnc(n, 1.0), hnr(n, 1.0);   // running norms
    Accum tb(n), tc(n), ttb(n), ttc(n);

    for (int r = 1; r < n; ++r) {
        // t_b = H b over the strictly upper column r of A (prec.cpp:366-381)
        for (int q = up[r]; q < up[r + 1]; ++q)
            for (const Entry &e : ht[urow[q]]) tb.add(e.idx, uval[q] * e.v);
        drop(tb, idv, dtol1, gnc, limit, filtit, coeff);
        tb.walk([&](int k) {
            if (std::fabs(tb.val[k]) != 0.0) ut[k].push_back({r, idv[k] * tb.val[k]});
        });
        // tt_b = G D^{-1} t_b (prec.cpp:450-474)
        tb.walk([&](int k) {
            const double t = tb.val[k];
            if (std::fabs(t) != 0.0)
                for (const Entry &e : gcol[k]) ttb.add(e.idx, t * idv[k] * e.v);
        });
        // t_c = c G over the strictly lower row r of A (prec.cpp:478-532)
        for (int q = lp[r]; q < lp[r + 1]; ++q)
            for (const Entry &e : gt[lcol[q]]) tc.add(e.idx, lval[q] * e.v);
        drop(tc, idv, dtol1, hnr, limit, filtit, coeff);
        tc.walk([&](int k) {
            if (std::fabs(tc.val[k]) != 0.0) lt[k].push_back({r, idv[k] * tc.val[k]});
        });
        // tt_c = t_c D^{-1} H (prec.cpp:599-622)
        tc.walk([&](int k) {
            const double t = tc.val[k];
            if (std::fabs(t) != 0.0)
                for (const Entry &e : hrow[k]) ttc.add(e.idx, idv[k] * t * e.v);
        });
        // s = d + t_b^T D^{-1} t_c, walking t_b's chain (prec.cpp:624-646)
        const double dr = d[r];
        double sum = 0.0;
        tb.walk([&](int k) { sum += tb.val[k] * idv[k] * tc.val[k]; });
        tb.clear();
        tc.clear();
        double s = dr + sum;
        // s1 = -c g_r, and the running column norm of g (prec.cpp:648-656)
        double s1 = 0.0;
        for (int q = lp[r]; q < lp[r + 1]; ++q) {
            const int k = lcol[q];
            s1 -= lval[q] * ttb.val[k];
            const double a = std::fabs(ttb.val[k]);
            gnc[r] = gnc[r] > a ? gnc[r] : a;
        }
        // g_r: norms updated on the first pass only, then the drop filter (prec.cpp:658-713)
        {
            int cut = 0;
            ttb.walk([&](int k) {
                gn[k] = gn[k] + std::fabs(ttb.val[k]);
                if (std::fabs(ttb.val[k]) <= dtol2 * gn[k]) {
                    ttb.val[k] = 0.0;
                    ++cut;
                }
            });
            double mult = 1.0;
            for (int l = 1; ttb.count - cut > limit && l <= filtit; ++l) {
                cut = 0;
                ttb.walk([&](int k) {
                    if (std::fabs(ttb.val[k]) <= mult * dtol2 * gn[k]) {
                        ttb.val[k] = 0.0;
                        ++cut;
                    }
                });
                mult *= coeff;
            }
            List &g = gcol[r];
            g.reserve(ttb.count - cut + 1);
            ttb.walk([&](int k) {
                if (ttb.val[k] != 0.0) g.push_back({k, -ttb.val[k]});
            });
            g.push_back({r, 1.0});
            ttb.clear();
        }
        // s2 = -h_r b, and the running row norm of h (prec.cpp:715-723)
        double s2 = 0.0;
        for (int q = up[r]; q < up[r + 1]; ++q) {
            const int k = urow[q];
            s2 -= uval[q] * ttc.val[k];
            const double a = std::fabs(ttc.val[k]);
            hnr[r] = hnr[r] > a ? hnr[r] : a;
        }
        // h_r, as g_r (prec.cpp:725-780)
        {
            int cut = 0;
            ttc.walk([&](int k) {
                hn[k] = hn[k] + std::fabs(ttc.val[k]);
                if (std::fabs(ttc.val[k]) <= dtol2 * hn[k]) {
                    ttc.val[k] = 0.0;
                    ++cut;
                }
            });
            double mult = 1.0;
            for (int l = 1; ttc.count - cut > limit && l <= filtit; ++l) {
                cut = 0;
                ttc.walk([&](int k) {
                    if (std::fabs(ttc.val[k]) <= mult * dtol2 * hn[k]) {
                        ttc.val[k] = 0.0;
                        ++cut;
                    }
                });
                mult *= coeff;
            }
            List &h = hrow[r];
            h.reserve(ttc.count - cut + 1);
            ttc.walk([&](int k) {
                if (ttc.val[k] != 0.0) h.push_back({k, -ttc.val[k]});
            });
            h.push_back({r, 1.0});
            ttc.clear();
        }
        for (const Entry &e : gcol[r]) gt[e.idx].push_back({r, e.v});
        for (const Entry &e : hrow[r]) ht[e.idx].push_back({r, e.v});
        // pivot (prec.cpp:830-836)
        s += (s1 + s2) + shift * std::fabs(dr);
        if (std::isnan(s)) return fiim::set_error(FIIM_EARG, "acifim: the Schur complement of row %d is NaN", r);
        if (std::fabs(s) <= eta) s = 1e-4 + dtol2;
        idv[r] = 1. / s;
    }
    out.n = n;
    rows_of(gt, out.Gi, out.Gj, out.Gv);
    rows_of(ut, out.Ui, out.Uj, out.Uv);
    rows_of_transposed(ht, out.Hi, out.Hj, out.Hv);
    rows_of_transposed(lt, out.Li, out.Lj, out.Lv);
    return FIIM_OK;
}

thread_local Factors g_acifim;

template <class T>
void put(const std::vector<T> &v, T *dst) {
    if (dst && !v.empty()) std::memcpy(dst, v.data(), sizeof(T) * v.size());
}

}  // namespace

extern "C" int fiim_acifim_build(int n, const int *Ai, const int *Aj, const double *Av, double dtol1, double dtol2,
                                 int elemPerRowCol, int growth, double eta, double shift, double coeff,
                                 int element_limit, int filtit, int *nnz, double *Gv, int *Gj, int *Gi, double *IDv,
                                 double *Hv, int *Hj, int *Hi, double *Lv, int *Lj, int *Li, double *Uv, int *Uj,
                                 int *Ui) {
    (void)elemPerRowCol;
    (void)growth;
    if (!Gv) {
        if (n <= 0 || !Ai || !Aj || !Av || !nnz) return fiim::set_error(FIIM_EARG, "acifim: need n > 0, A and nnz");
        g_acifim = Factors();
        const int rc = build(n, Ai, Aj, Av, dtol1, dtol2, eta, shift, coeff, element_limit, filtit, g_acifim);
        if (rc != FIIM_OK) {
            g_acifim = Factors();
            return rc;
        }
        nnz[0] = g_acifim.Gi[n];
        nnz[1] = g_acifim.Hi[n];
        nnz[2] = g_acifim.Li[n];
        nnz[3] = g_acifim.Ui[n];
        return FIIM_OK;
    }
    if (g_acifim.n != n || !Gj || !Gi || !IDv || !Hv || !Hj || !Hi)
        return fiim::set_error(FIIM_EARG, "acifim: copy-out call without a matching sizing call");
    put(g_acifim.Gi, Gi);
    put(g_acifim.Gj, Gj);
    put(g_acifim.Gv, Gv);
    put(g_acifim.IDv, IDv);
    put(g_acifim.Hi, Hi);
    put(g_acifim.Hj, Hj);
    put(g_acifim.Hv, Hv);
    if (Lv && Lj && Li) {
        put(g_acifim.Li, Li);
        put(g_acifim.Lj, Lj);
        put(g_acifim.Lv, Lv);
    }
    if (Uv && Uj && Ui) {
        put(g_acifim.Ui, Ui);
        put(g_acifim.Uj, Uj);
        put(g_acifim.Uv, Uv);
    }
    g_acifim = Factors();
    return FIIM_OK;
}
