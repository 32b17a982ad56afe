// AFIIM factor construction on the host: the same G, D^{-1}, H as afiim
// (AFIIM/src/prec.cpp:101-767), bit for bit, for callers and benchmarks that need AFIIM
// factors without the reference library.
//
// The sweep is ACIFIM's (fiim_acifim.cpp) without the stored L and U and without repeated
// filter passes: for r = 1 .. n-1, t_b = H b and t_c = c G over the strictly upper column
// and strictly lower row r of A, g_r = -G D^{-1} t_b and h_r = -t_c D^{-1} H, each entry
// dropped when |g_rk| <= eps |g|_k / min(|u_r|, |a_r|) (running column maxima of G, the
// largest |D^{-1} t_b| of this step, and the row maximum of A's strictly lower part scaled
// by sqrt|d_i d_j|; the mirror image for h_r), and s_r = d_r + t_b^T D^{-1} t_c - c g_r - h_r b.
// Sums run in the reference's order (accumulators walked newest index first) and products
// left to right as written there; compiled without FMA contraction. The sweep is sequential
// in r, as the reference's is: one system per call (and per thread).

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

inline double vmax(double a, double b) { return a > b ? a : b; }
inline double vmin(double a, double b) { return a < b ? a : b; }

int build(int n, const int *Ai, const int *Aj, const double *Av, double dtol, double eta, double shift,
          Factors &out) {
    fiim::sweep::Split a;
    fiim::sweep::split(n, Ai, Aj, Av, dtol, a);
    const std::vector<double> &d = a.d, &lval = a.lval, &uval = a.uval;
    const std::vector<int> &lp = a.lp, &lcol = a.lcol, &up = a.up, &urow = a.urow;
    // Largest |a_ij| / (sqrt|d_i| sqrt|d_j|) of each strictly upper column and strictly lower
    // row of A, at least 1 (prec.cpp:308-327).
    std::vector<double> auc(n, 1.0), alr(n, 1.0);
    for (int i = 0; i < n; ++i)
        for (int q = up[i]; q < up[i + 1]; ++q)
            auc[i] = vmax(auc[i], std::fabs(uval[q]) / (std::sqrt(std::fabs(d[i])) * std::sqrt(std::fabs(d[urow[q]]))));
    for (int i = 0; i < n; ++i)
        for (int q = lp[i]; q < lp[i + 1]; ++q)
            alr[i] = vmax(alr[i], std::fabs(lval[q]) / (std::sqrt(std::fabs(d[i])) * std::sqrt(std::fabs(d[lcol[q]]))));

    std::vector<double> &idv = out.IDv;
    idv.assign(n, 0.0);
    {
        const double s = d[0] + shift * std::fabs(d[0]);
        idv[0] = (std::fabs(s) < eta) ? 1.0 / (1e-4 + dtol) : 1.0 / s;
    }
    std::vector<List> gcol(n), hrow(n), gt(n), ht(n);
    gcol[0] = {{0, 1.0}};
    hrow[0] = {{0, 1.0}};
    gt[0] = {{0, 1.0}};
    ht[0] = {{0, 1.0}};
    std::vector<double> gn(n, 1.0), hn(n, 1.0), un(n, 1.0), ln(n, 1.0);   // running maxima
    Accum tb(n), tc(n), ttb(n), ttc(n);

    for (int r = 1; r < n; ++r) {
        // t_b = H b (prec.cpp:357-377); tt_b = G D^{-1} t_b and the step's |D^{-1} t_b| max
        for (int q = up[r]; q < up[r + 1]; ++q)
            for (const Entry &e : ht[urow[q]]) tb.add(e.idx, uval[q] * e.v);
        tb.walk([&](int k) {
            for (const Entry &e : gcol[k]) ttb.add(e.idx, tb.val[k] * idv[k] * e.v);
            un[r] = vmax(un[r], std::fabs(idv[k] * tb.val[k]));
        });
        // t_c = c G (prec.cpp:405-425); tt_c = t_c D^{-1} H and the step's |t_c D^{-1}| max
        for (int q = lp[r]; q < lp[r + 1]; ++q)
            for (const Entry &e : gt[lcol[q]]) tc.add(e.idx, lval[q] * e.v);
        tc.walk([&](int k) {
            for (const Entry &e : hrow[k]) ttc.add(e.idx, idv[k] * tc.val[k] * e.v);
            ln[r] = vmax(ln[r], std::fabs(tc.val[k] * idv[k]));
        });
        // s = d + t_b^T D^{-1} t_c, walking t_b's chain (prec.cpp:452-476)
        const double dr = d[r];
        double sum = 0.0;
        tb.walk([&](int k) { sum += tb.val[k] * idv[k] * tc.val[k]; });
        tb.clear();
        tc.clear();
        double s = dr + sum;
        double s1 = 0.0;
        for (int q = lp[r]; q < lp[r + 1]; ++q) s1 -= lval[q] * ttb.val[lcol[q]];
        // g_r (prec.cpp:487-527)
        {
            const double m = vmin(un[r], alr[r]);
            ttb.walk([&](int k) {
                gn[k] = vmax(gn[k], std::fabs(ttb.val[k]));
                if (std::fabs(ttb.val[k]) <= dtol * gn[k] / m) ttb.val[k] = 0.0;
            });
            List &g = gcol[r];
            ttb.walk([&](int k) {
                if (ttb.val[k] != 0.0) g.push_back({k, -ttb.val[k]});
            });
            g.push_back({r, 1.0});
            ttb.clear();
        }
        double s2 = 0.0;
        for (int q = up[r]; q < up[r + 1]; ++q) s2 -= uval[q] * ttc.val[urow[q]];
        // h_r (prec.cpp:538-577)
        {
            const double m = vmin(ln[r], auc[r]);
            ttc.walk([&](int k) {
                hn[k] = vmax(hn[k], std::fabs(ttc.val[k]));
                if (std::fabs(ttc.val[k]) <= dtol * hn[k] / m) ttc.val[k] = 0.0;
            });
            List &h = hrow[r];
            ttc.walk([&](int k) {
                if (ttc.val[k] != 0.0) h.push_back({k, -ttc.val[k]});
            });
            h.push_back({r, 1.0});
            ttc.clear();
        }
        for (const Entry &e : gcol[r]) gt[e.idx].push_back({r, e.v});
        for (const Entry &e : hrow[r]) ht[e.idx].push_back({r, e.v});
        // pivot (prec.cpp:634-637)
        s += (s1 + s2) + shift * std::fabs(dr);
        if (std::fabs(s) <= eta) s = 1e-4 + dtol;
        idv[r] = 1. / s;
    }
    out.n = n;
    fiim::sweep::rows_of(gt, out.Gi, out.Gj, out.Gv);
    fiim::sweep::rows_of_transposed(ht, out.Hi, out.Hj, out.Hv);
    return FIIM_OK;
}

thread_local Factors g_afiim;

template <class T>
void put(const std::vector<T> &v, T *dst) {
    if (dst && !v.empty()) std::memcpy(dst, v.data(), sizeof(T) * v.size());
}

}  // namespace

extern "C" int fiim_afiim_build(int n, const int *Ai, const int *Aj, const double *Av, double dtol, int elemPerRowCol,
                                int growth, double eta, double shift, int *nnzG, int *nnzH, double *Gv, int *Gj,
                                int *Gi, double *IDv, double *Hv, int *Hj, int *Hi) {
    (void)elemPerRowCol;
    (void)growth;
    if (!Gv) {
        if (n <= 0 || !Ai || !Aj || !Av || !nnzG || !nnzH)
            return fiim::set_error(FIIM_EARG, "afiim: need n > 0, A, nnzG and nnzH");
        g_afiim = Factors();
        const int rc = build(n, Ai, Aj, Av, dtol, eta, shift, g_afiim);
        if (rc != FIIM_OK) {
            g_afiim = Factors();
            return rc;
        }
        *nnzG = g_afiim.Gi[n];
        *nnzH = g_afiim.Hi[n];
        return FIIM_OK;
    }
    if (g_afiim.n != n || !Gj || !Gi || !IDv || !Hv || !Hj || !Hi)
        return fiim::set_error(FIIM_EARG, "afiim: copy-out call without a matching sizing call");
    put(g_afiim.Gi, Gi);
    put(g_afiim.Gj, Gj);
    put(g_afiim.Gv, Gv);
    put(g_afiim.IDv, IDv);
    put(g_afiim.Hi, Hi);
    put(g_afiim.Hj, Hj);
    put(g_afiim.Hv, Hv);
    g_afiim = Factors();
    return FIIM_OK;
}
