// Synthetic problem generators for the solve phase's workloads. The reference ships
// no generators (its only fixture is HB/sherman2); these produce 0-based CSR with
// ascending column indices inside each row, the layout the reference's Matrix Market
// reader emits (AFIIM/src/rw_matrix.cpp:186-210) and that PDFIIM's construction
// assumes (PDFIIM/src/parPrec.cpp:132 reads the first entry of row 0 as its diagonal).
//
// Every generator has a sizing pass: call with null output arrays to get nnz.
// Random draws use splitmix64 so that the same seed gives the same matrix on any host.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

#include "fiim_b200.h"

namespace {

inline uint64_t splitmix64(uint64_t &s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
// Uniform in [0,1) with 53 random bits.
inline double unif(uint64_t &s) { return (double)(splitmix64(s) >> 11) * (1.0 / 9007199254740992.0); }
// Standard normal by the Box-Muller transform.
inline double normal(uint64_t &s) {
    double u1 = unif(s), u2 = unif(s);
    if (u1 < 1e-300) u1 = 1e-300;
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}
// Independent stream per (seed, index).
inline uint64_t stream_seed(uint64_t seed, uint64_t idx) {
    uint64_t s = seed ^ (0xD1B54A32D192ED03ull * (idx + 1));
    splitmix64(s);
    return s;
}

struct Entry { int col; double val; };

}  // namespace

extern "C" {

long fiim_gen_poisson2d(int nx, int ny, int *Ai, int *Aj, double *Av) {
    if (nx <= 0 || ny <= 0) return -1;
    const long n = (long)nx * ny;
    const long nnz = 5 * n - 2L * nx - 2L * ny;
    if (!Ai) return nnz;
    long c = 0;
    Ai[0] = 0;
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            const long i = x + (long)nx * y;
            if (y > 0) { Aj[c] = (int)(i - nx); Av[c++] = -1.0; }
            if (x > 0) { Aj[c] = (int)(i - 1); Av[c++] = -1.0; }
            Aj[c] = (int)i; Av[c++] = 4.0;
            if (x < nx - 1) { Aj[c] = (int)(i + 1); Av[c++] = -1.0; }
            if (y < ny - 1) { Aj[c] = (int)(i + nx); Av[c++] = -1.0; }
            Ai[i + 1] = (int)c;
        }
    return c;
}

// -div(grad u) + v . grad(u) on an N^3 grid, Dirichlet boundary, unit diffusion,
// velocity (c,c,c) with cell Peclet number c*h/1 = peclet, first-order upwind, scaled
// by h^2: diagonal 6 + 3*peclet, upwind (lower) neighbours -1 - peclet, others -1.
long fiim_gen_convdiff3d(int N, double peclet, int *Ai, int *Aj, double *Av) {
    if (N <= 0) return -1;
    const long n = (long)N * N * N;
    const long nnz = 7 * n - 6L * N * N;
    if (!Ai) return nnz;
    if (n > 0x7fffffffL || nnz > 0x7fffffffL) return -2;
    const double dg = 6.0 + 3.0 * peclet, lo = -1.0 - peclet, hi = -1.0;
    const long NN = (long)N * N;
    Ai[0] = 0;
    for (long i = 0; i < n; ++i) {   // row offsets: count, then fill in parallel
        const int x = (int)(i % N), y = (int)((i / N) % N), z = (int)(i / NN);
        int len = 1 + (x > 0) + (x < N - 1) + (y > 0) + (y < N - 1) + (z > 0) + (z < N - 1);
        Ai[i + 1] = Ai[i] + len;
    }
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) {
        const int x = (int)(i % N), y = (int)((i / N) % N), z = (int)(i / NN);
        long c = Ai[i];
        if (z > 0) { Aj[c] = (int)(i - NN); Av[c++] = lo; }
        if (y > 0) { Aj[c] = (int)(i - N); Av[c++] = lo; }
        if (x > 0) { Aj[c] = (int)(i - 1); Av[c++] = lo; }
        Aj[c] = (int)i; Av[c++] = dg;
        if (x < N - 1) { Aj[c] = (int)(i + 1); Av[c++] = hi; }
        if (y < N - 1) { Aj[c] = (int)(i + N); Av[c++] = hi; }
        if (z < N - 1) { Aj[c] = (int)(i + NN); Av[c++] = hi; }
    }
    return nnz;
}

// -d*lap(u) + v . grad(u) on an N x N grid, Dirichlet boundary, first-order upwind,
// scaled by h^2, with v = |v| (cos t, sin t) and |v| h / d = peclet.
long fiim_gen_convdiff2d(int N, double diff, double theta, double peclet, int *Ai, int *Aj,
                         double *Av) {
    if (N <= 0 || !(diff > 0)) return -1;
    const long n = (long)N * N;
    const long nnz = 5 * n - 4L * N;
    if (!Ai) return nnz;
    const double vh = peclet * diff;                 // |v| * h
    const double cx = vh * std::cos(theta), cy = vh * std::sin(theta);
    const double west = -diff - (cx > 0 ? cx : 0.0), east = -diff - (cx < 0 ? -cx : 0.0);
    const double south = -diff - (cy > 0 ? cy : 0.0), north = -diff - (cy < 0 ? -cy : 0.0);
    const double dg = 4.0 * diff + std::fabs(cx) + std::fabs(cy);
    long c = 0;
    Ai[0] = 0;
    for (int y = 0; y < N; ++y)
        for (int x = 0; x < N; ++x) {
            const long i = x + (long)N * y;
            if (y > 0) { Aj[c] = (int)(i - N); Av[c++] = south; }
            if (x > 0) { Aj[c] = (int)(i - 1); Av[c++] = west; }
            Aj[c] = (int)i; Av[c++] = dg;
            if (x < N - 1) { Aj[c] = (int)(i + 1); Av[c++] = east; }
            if (y < N - 1) { Aj[c] = (int)(i + N); Av[c++] = north; }
            Ai[i + 1] = (int)c;
        }
    return c;
}

// Parameters of system k of the batched 2D family: grid side U{side_lo..side_hi},
// diffusion log-uniform in [d_lo, d_hi], direction U[0, 2pi), cell Peclet U(0, pe_max].
void fiim_gen_batch_params(uint64_t seed, int k, int side_lo, int side_hi, double d_lo,
                           double d_hi, double pe_max, int *side, double *diff, double *theta,
                           double *peclet) {
    uint64_t s = stream_seed(seed, (uint64_t)k);
    *side = side_lo + (int)(splitmix64(s) % (uint64_t)(side_hi - side_lo + 1));
    *diff = std::exp(std::log(d_lo) + unif(s) * (std::log(d_hi) - std::log(d_lo)));
    *theta = 6.283185307179586 * unif(s);
    *peclet = pe_max * (1.0 - unif(s));
}

// Random nonsymmetric matrix: row lengths round(scale * Z) clipped to [1, cap] with
// Z ~ Zipf(alpha) truncated to [1, cap]; distinct uniform columns plus the diagonal;
// off-diagonal values U(-1,1); diagonal 1.1 x the absolute off-diagonal row sum.
// `scale` is chosen by the caller (fiim_gen_zipf_scale) to hit a target mean.
long fiim_gen_zipf(int n, double alpha, int cap, double scale, uint64_t seed, int *Ai, int *Aj,
                   double *Av) {
    if (n <= 0 || cap < 1) return -1;
    // Inverse-CDF table for the truncated Zipf law.
    std::vector<double> cdf(cap);
    double z = 0.0;
    for (int k = 1; k <= cap; ++k) { z += std::pow((double)k, -alpha); cdf[k - 1] = z; }
    for (auto &v : cdf) v /= z;
    auto row_len = [&](long i) {
        uint64_t s = stream_seed(seed, (uint64_t)i);
        const double u = unif(s);
        const int k = (int)(std::lower_bound(cdf.begin(), cdf.end(), u) - cdf.begin()) + 1;
        long len = std::lround(scale * k);
        if (len < 1) len = 1;
        if (len > cap) len = cap;
        if (len > n) len = n;
        return (int)len;       // includes the diagonal
    };
    if (!Ai) {
        long nnz = 0;
#pragma omp parallel for reduction(+ : nnz) schedule(static)
        for (long i = 0; i < n; ++i) nnz += row_len(i);
        return nnz;
    }
    Ai[0] = 0;
    for (long i = 0; i < n; ++i) Ai[i + 1] = Ai[i] + row_len(i);
#pragma omp parallel
    {
        std::vector<int> cols;
#pragma omp for schedule(dynamic, 4096)
        for (long i = 0; i < n; ++i) {
            const int len = Ai[i + 1] - Ai[i];
            uint64_t s = stream_seed(seed ^ 0x5bd1e995ull, (uint64_t)i);
            cols.clear();
            cols.push_back((int)i);
            while ((int)cols.size() < len) {
                const int c = (int)(splitmix64(s) % (uint64_t)n);
                if (std::find(cols.begin(), cols.end(), c) == cols.end()) cols.push_back(c);
            }
            std::sort(cols.begin(), cols.end());
            double asum = 0.0;
            long d = -1;
            for (int k = 0; k < len; ++k) {
                const long o = Ai[i] + k;
                Aj[o] = cols[k];
                if (cols[k] == i) { d = o; continue; }
                Av[o] = 2.0 * unif(s) - 1.0;
                asum += std::fabs(Av[o]);
            }
            Av[d] = 1.1 * asum > 0 ? 1.1 * asum : 1.0;
        }
    }
    return Ai[n];
}

// Mean row length of fiim_gen_zipf for a given scale, over the first `sample` rows.
double fiim_gen_zipf_mean(int n, double alpha, int cap, double scale, uint64_t seed, int sample) {
    std::vector<double> cdf(cap);
    double z = 0.0;
    for (int k = 1; k <= cap; ++k) { z += std::pow((double)k, -alpha); cdf[k - 1] = z; }
    for (auto &v : cdf) v /= z;
    const int m = sample < n ? sample : n;
    double tot = 0.0;
    for (long i = 0; i < m; ++i) {
        uint64_t s = stream_seed(seed, (uint64_t)i);
        const double u = unif(s);
        const int k = (int)(std::lower_bound(cdf.begin(), cdf.end(), u) - cdf.begin()) + 1;
        long len = std::lround(scale * k);
        if (len < 1) len = 1;
        if (len > cap) len = cap;
        if (len > n) len = n;
        tot += (double)len;
    }
    return tot / m;
}

void fiim_rand_normal(long n, uint64_t seed, double *out) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) {
        uint64_t s = stream_seed(seed, (uint64_t)i);
        out[i] = normal(s);
    }
}

// b = A * 1 (the reference's model right-hand side, AFIIM/src/misc.cpp:51-74).
void fiim_model_rhs(int n, const int *Ai, const int *Aj, const double *Av, double *b) {
    (void)Aj;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) {
        double s = 0.0;
        for (int k = Ai[i]; k < Ai[i + 1]; ++k) s += Av[k];
        b[i] = s;
    }
}

}  // extern "C"
