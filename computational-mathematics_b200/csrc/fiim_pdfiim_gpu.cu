// PDFIIM factor construction on the GPU: the same G, D^{-1} and H as the host construction
// (fiim_pdfiim.cpp), and so as the reference's pdfiim (PDFIIM/src/parPrec.cpp:95-588) for
// pattern 'B', bit for bit. One warp builds one row i at a time:
//   * the row's pattern, an insertion-ordered set, lives in the warp's shared memory; a
//     row of A or A^T is merged into it 32 entries at a time, the absent columns appended in
//     column order (the same order as one-by-one insertion, since a row's columns are
//     distinct);
//   * the dense LU with partial pivoting of the pattern's B (Golub & Van Loan Alg. 3.4.1,
//     first largest pivot) eliminates one row per lane; every product and difference is
//     rounded separately, as the host code compiled without contraction;
//   * the assembly of the right-hand sides, the triangular solves, the filter norms and the
//     D^{-1} sums keep the host's sequential order (lane 0);
//   * kept entries are sorted by index through their ranks.
// Two passes over the rows: the first counts the kept entries of every row, the host turns
// the counts into offsets, the second writes the entries and D^{-1}. A row whose pattern
// outgrows the warp's shared memory (CAP members in a solve, 4 CAP in the set; 2048 at the
// largest CAP) is listed and built again with a larger CAP; past the largest CAP the call
// returns FIIM_EARG and the host construction serves.

#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <vector>

#include "fiim_b200.h"
#include "fiim_internal.h"
#include "fiim_kernels.cuh"

namespace fiim {
namespace pg {

struct CsrD {
    const int *rp, *ci;
    const double *v;
};

struct Params {
    int prefill, lfill, postfill, warpsize;
    double ftol;
    char filttype;
};

struct Out {
    int *gcnt, *hcnt;           // kept entries + unit diagonal, per row
    double *D;
    const long *goff, *hoff;    // write pass: entry offsets of each row
    int *gj, *hj;
    double *gv, *hv;
    int *overflow, *noverflow;  // rows left for a larger CAP
};

template <int CAP>
struct WarpSmem {
    // Set capacity: 4 CAP, and 2048 at the largest CAP, where a warpsize cap keeps the solve
    // small while wide rows (random columns, hundreds of entries) still grow the set.
    static constexpr int SET = CAP >= 128 ? 2048 : 4 * CAP;
    int list[SET];
    int inds[CAP];
    int piv[CAP];
    int rank[CAP];
    double g[CAP], h[CAP];
    double B[CAP * CAP];
};

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

template <int CAP>
struct RowBuilder {
    WarpSmem<CAP> &s;
    const CsrD &A, &At;
    const int i, lane;
    int size = 0;
    bool over = false;

    __device__ RowBuilder(WarpSmem<CAP> &s_, const CsrD &A_, const CsrD &At_, int i_)
        : s(s_), A(A_), At(At_), i(i_), lane((int)(threadIdx.x & 31)) {}

    // Columns < i of row j of M, appended in column order where absent.
    __device__ void push_row_below(const CsrD &M, int j) {
        if (over) return;
        const int beg = M.rp[j], end = M.rp[j + 1];
        for (int base = beg; base < end; base += 32) {
            const int k = base + lane;
            const int c = k < end ? M.ci[k] : INT_MAX;
            const bool valid = c < i;
            bool present = false;
            if (valid)
                for (int q = 0; q < size; ++q)
                    if (s.list[q] == c) {
                        present = true;
                        break;
                    }
            const unsigned add = __ballot_sync(0xffffffffu, valid && !present);
            if (valid && !present) {
                const int at = size + __popc(add & lanemask_lt());
                if (at < WarpSmem<CAP>::SET) s.list[at] = c;
            }
            size += __popc(add);
            if (size > WarpSmem<CAP>::SET) over = true;
            __syncwarp();
            if (!__all_sync(0xffffffffu, valid) || over) break;
        }
    }

    __device__ int pos_of(int c, int len) const {
        for (int q = 0; q < len; ++q)
            if (s.inds[q] == c) return q;
        return -1;
    }

    // LU with partial pivoting of B (len x len, row-major), then B g = g, B^T h = h.
    __device__ void factor_solve(int len) {
        double *B = s.B;
        for (int k = 0; k < len; ++k) {
            // First row of largest |B(r, k)|, r >= k, as a sequential scan from r = k finds it
            // (a NaN at (k, k) keeps row k, a NaN below is never taken).
            double best = -1.0;
            int p = len;
            for (int r = k + lane; r < len; r += 32) {
                const double v = fabs(B[r * len + k]);
                if (v > best) {
                    best = v;
                    p = r;
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int op = __shfl_xor_sync(0xffffffffu, p, o);
                if (ob > best || (ob == best && op < p)) {
                    best = ob;
                    p = op;
                }
            }
            if (isnan(B[k * len + k])) p = k;
            if (lane == 0) s.piv[k] = p;
            __syncwarp();
            if (B[p * len + k] == 0.0) continue;
            if (p != k)
                for (int c = lane; c < len; c += 32) {
                    const double t = B[k * len + c];
                    B[k * len + c] = B[p * len + c];
                    B[p * len + c] = t;
                }
            __syncwarp();
            const double d = B[k * len + k];
            for (int r = k + 1 + lane; r < len; r += 32) {
                const double l = B[r * len + k] / d;
                B[r * len + k] = l;
                for (int c = k + 1; c < len; ++c)
                    B[r * len + c] = __dsub_rn(B[r * len + c], __dmul_rn(l, B[k * len + c]));
            }
            __syncwarp();
        }
        if (lane == 0) {
            double *g = s.g, *h = s.h;
            const int *piv = s.piv;
            // B g = g: row swaps, forward, backward (lu_solve)
            for (int k = 0; k < len; ++k)
                if (piv[k] != k) {
                    const double t = g[k];
                    g[k] = g[piv[k]];
                    g[piv[k]] = t;
                }
            for (int r = 0; r < len; ++r) {
                double acc = g[r];
                for (int c = 0; c < r; ++c) acc = __dsub_rn(acc, __dmul_rn(B[r * len + c], g[c]));
                g[r] = acc;
            }
            for (int r = len - 1; r >= 0; --r) {
                double acc = g[r];
                for (int c = r + 1; c < len; ++c) acc = __dsub_rn(acc, __dmul_rn(B[r * len + c], g[c]));
                g[r] = acc / B[r * len + r];
            }
            // B^T h = h (lu_solve_t)
            for (int r = 0; r < len; ++r) {
                double acc = h[r];
                for (int c = 0; c < r; ++c) acc = __dsub_rn(acc, __dmul_rn(B[c * len + r], h[c]));
                h[r] = acc / B[r * len + r];
            }
            for (int r = len - 1; r >= 0; --r) {
                double acc = h[r];
                for (int c = r + 1; c < len; ++c) acc = __dsub_rn(acc, __dmul_rn(B[c * len + r], h[c]));
                h[r] = acc;
            }
            for (int k = len - 1; k >= 0; --k)
                if (piv[k] != k) {
                    const double t = h[k];
                    h[k] = h[piv[k]];
                    h[piv[k]] = t;
                }
        }
        __syncwarp();
    }
};

__device__ double filter_norm(char filttype, const double *x, int len) {
    double nrm = 1.0;
    if (filttype == '1') {
        for (int j = 0; j < len; ++j) nrm = __dadd_rn(nrm, fabs(x[j]));
        nrm = nrm / (double)(len + 1);
    } else if (filttype == '2') {
        for (int j = 0; j < len; ++j) nrm = __dadd_rn(nrm, __dmul_rn(x[j], x[j]));
        nrm = sqrt(nrm);
    } else {
        for (int j = 0; j < len; ++j) nrm = (nrm < fabs(x[j])) ? fabs(x[j]) : nrm;
    }
    return nrm;
}

// Rows rows[0..nrows) (or 1..n-1 when rows == NULL), one warp each.
template <int CAP, bool WRITE>
static __global__ void __launch_bounds__(256)
k_pdfiim_rows(int n, const int *__restrict__ rows, int nrows, CsrD A, CsrD At, Params P, Out o) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    WarpSmem<CAP> &s = reinterpret_cast<WarpSmem<CAP> *>(smem_raw)[w];
    const long wid = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long nw = ((long)gridDim.x * blockDim.x) >> 5;
    const long total = rows ? nrows : (long)n - 1;
    const double floor_diag = fmax(1e-4, P.ftol);
    for (long t = wid; t < total; t += nw) {
        const int i = rows ? rows[t] : (int)(t + 1);
        RowBuilder<CAP> rb(s, A, At, i);
        // Level 1 and the pre-fill levels (parPrec.cpp:144-177), newest member first.
        rb.push_row_below(At, i);
        rb.push_row_below(A, i);
        for (int k = 2; k <= P.prefill && !rb.over; ++k) {
            const int len = rb.size;
            for (int q = len - 1; q >= 0 && !rb.over; --q) {
                const int jind = s.list[q];
                rb.push_row_below(At, jind);
                rb.push_row_below(A, jind);
            }
        }
        int tlen = 0;
        double ng = 0.0, nh = 0.0;
        for (int k = 1; k <= P.lfill && !rb.over; ++k) {
            ng = 0.0;
            int len = rb.size;
            tlen = len;
            if (len == 0) break;
            if (P.warpsize != -1)
                for (int j = len; j >= P.warpsize; --j) rb.size--;   // drop the newest members
            len = rb.size;
            tlen = len;
            if (len > CAP) {
                rb.over = true;
                break;
            }
            __syncwarp();
            for (int j = lane; j < len; j += 32) s.inds[j] = s.list[j];
            for (int q = lane; q < len * len; q += 32) s.B[q] = 0.0;
            for (int j = lane; j < len; j += 32) {
                s.g[j] = 0.0;
                s.h[j] = 0.0;
            }
            __syncwarp();
            // B = A restricted to the pattern (one row per lane, in storage order), with the
            // diagonal floor.
            for (int j = lane; j < len; j += 32) {
                const int row = s.inds[j];
                s.B[j * len + j] = floor_diag;
                for (int kk = A.rp[row]; kk < A.rp[row + 1] && A.ci[kk] < i; ++kk) {
                    const int q = rb.pos_of(A.ci[kk], len);
                    if (q >= 0) s.B[j * len + q] = A.v[kk];
                }
                if (s.B[j * len + j] == 0.0) s.B[j * len + j] = floor_diag;
            }
            __syncwarp();
            if (lane == 0) {   // g from A^T row i, h from A row i, in storage order
                for (int kk = At.rp[i]; kk < At.rp[i + 1]; ++kk)
                    if (At.ci[kk] < i) {
                        const int q = rb.pos_of(At.ci[kk], len);
                        if (q >= 0) s.g[q] = -At.v[kk];
                    }
                for (int kk = A.rp[i]; kk < A.rp[i + 1]; ++kk)
                    if (A.ci[kk] < i) {
                        const int q = rb.pos_of(A.ci[kk], len);
                        if (q >= 0) s.h[q] = -A.v[kk];
                    }
            }
            __syncwarp();
            rb.factor_solve(len);
            ng = __shfl_sync(0xffffffffu, lane == 0 ? filter_norm(P.filttype, s.g, len) : 0.0, 0);
            nh = __shfl_sync(0xffffffffu, lane == 0 ? filter_norm(P.filttype, s.h, len) : 0.0, 0);
            // New set: kept g entries in order, then kept h entries not yet in it.
            rb.size = 0;
            int c = 0, c2 = 0;
            for (int base = 0; base < len; base += 32) {
                const int j = base + lane;
                const bool kg = j < len && fabs(s.g[j]) >= P.ftol * ng;
                const unsigned m = __ballot_sync(0xffffffffu, kg);
                if (kg) s.list[rb.size + __popc(m & lanemask_lt())] = s.inds[j];
                rb.size += __popc(m);
                c += __popc(m);
            }
            for (int base = 0; base < len; base += 32) {
                const int j = base + lane;
                const bool kh = j < len && fabs(s.h[j]) >= P.ftol * nh;
                const bool kg = j < len && fabs(s.g[j]) >= P.ftol * ng;
                const unsigned mh = __ballot_sync(0xffffffffu, kh);
                const unsigned m = __ballot_sync(0xffffffffu, kh && !kg);
                if (kh && !kg) s.list[rb.size + __popc(m & lanemask_lt())] = s.inds[j];
                rb.size += __popc(m);
                c2 += __popc(mh);
            }
            __syncwarp();
            if ((c == 0 && c2 == 0) || c2 == P.warpsize) break;
            // The last level's growth reaches nothing the result depends on.
            if (k == P.lfill) break;
            // Next level set from the first |set| members of the solved pattern (parPrec.cpp:366-385).
            const int kept = rb.size;
            for (int j = 0; j < kept && !rb.over; ++j) {
                const int jind = s.inds[j];
                rb.push_row_below(At, jind);
                rb.push_row_below(A, jind);
            }
            for (int m = 2; m <= P.postfill && !rb.over; ++m) {
                const int len2 = rb.size;
                for (int q = len2 - 1; q >= 0 && !rb.over; --q) {
                    const int jind = s.list[q];
                    rb.push_row_below(At, jind);
                    rb.push_row_below(A, jind);
                }
            }
            if (rb.size == kept) break;
        }
        if (rb.over) {
            if (!WRITE && lane == 0) o.overflow[atomicAdd(o.noverflow, 1)] = i;
            __syncwarp();
            continue;
        }
        // Kept entries sorted by index (ranks), unit diagonal last (parPrec.cpp:460-500).
        int cnt[2] = {0, 0};
        for (int which = 0; which < 2; ++which) {
            const double *x = which == 0 ? s.g : s.h;
            const double nrm = which == 0 ? ng : nh;
            for (int j = lane; j < tlen; j += 32) {
                int r = -1;
                if (fabs(x[j]) >= P.ftol * nrm) {
                    r = 0;
                    for (int q = 0; q < tlen; ++q)
                        if (fabs(x[q]) >= P.ftol * nrm && s.inds[q] < s.inds[j]) ++r;
                }
                s.rank[j] = r;
            }
            int kc = 0;
            for (int base = 0; base < tlen; base += 32) {
                const int j = base + lane;
                kc += __popc(__ballot_sync(0xffffffffu, j < tlen && fabs(x[j]) >= P.ftol * nrm));
            }
            cnt[which] = kc;
            __syncwarp();
            if (WRITE) {
                const long off = which == 0 ? o.goff[i] : o.hoff[i];
                int *oj = which == 0 ? o.gj : o.hj;
                double *ov = which == 0 ? o.gv : o.hv;
                for (int j = lane; j < tlen; j += 32)
                    if (s.rank[j] >= 0) {
                        oj[off + s.rank[j]] = s.inds[j];
                        ov[off + s.rank[j]] = x[j];
                    }
                if (lane == 0) {
                    oj[off + kc] = i;
                    ov[off + kc] = 1.0;
                }
            }
            __syncwarp();
        }
        if (!WRITE) {
            if (lane == 0) {
                o.gcnt[i] = cnt[0] + 1;
                o.hcnt[i] = cnt[1] + 1;
            }
        } else if (lane == 0) {
            // D^{-1}_i = 1 / sum_j h_j (A g)_j over the kept patterns (parPrec.cpp:502-532).
            const long go = o.goff[i], ho = o.hoff[i];
            const int gn = cnt[0] + 1, hn = cnt[1] + 1;
            double sum = 0.0;
            for (int j = 0; j < hn; ++j) {
                const int hr = o.hj[ho + j];
                const double hvj = o.hv[ho + j];
                int kk = A.rp[hr], cc = 0;
                while (kk < A.rp[hr + 1] && cc < gn) {
                    const int gc = o.gj[go + cc];
                    if (A.ci[kk] == gc) {
                        sum = __dadd_rn(sum, __dmul_rn(__dmul_rn(hvj, A.v[kk]), o.gv[go + cc]));
                        ++kk;
                        ++cc;
                    } else if (A.ci[kk] < gc) {
                        ++kk;
                    } else {
                        ++cc;
                    }
                }
            }
            o.D[i] = 1.0 / sum;
        }
        __syncwarp();
    }
}

template <int CAP, bool WRITE>
int launch_rows(int n, const int *rows, int nrows, const CsrD &A, const CsrD &At, const Params &P, const Out &o,
                cudaStream_t st) {
    constexpr int warps = CAP <= 32 ? 8 : (CAP <= 64 ? 4 : 1);
    constexpr size_t smem = sizeof(WarpSmem<CAP>) * warps;
    auto kern = k_pdfiim_rows<CAP, WRITE>;
    FIIM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    FIIM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * warps, smem));
    const long total = rows ? nrows : (long)n - 1;
    const long need = (total + warps - 1) / warps;
    const int grid = (int)std::max<long>(1, std::min<long>(need, (long)std::max(per_sm, 1) * num_sms()));
    kern<<<grid, 32 * warps, smem, st>>>(n, rows, nrows, A, At, P, o);
    FIIM_CUDA(cudaGetLastError());
    return FIIM_OK;
}

struct DevBuf {
    std::vector<void *> ptrs;
    template <typename T>
    T *get(size_t count) {
        void *p = nullptr;
        if (cudaMalloc(&p, sizeof(T) * std::max<size_t>(count, 1)) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        ptrs.push_back(p);
        return static_cast<T *>(p);
    }
    ~DevBuf() {
        for (void *p : ptrs) cudaFree(p);
    }
};

struct BuiltGpu {
    int n = 0;
    std::vector<int> Gi, Gj, Hi, Hj;
    std::vector<double> Gv, Hv, D;
};
thread_local BuiltGpu g_built_gpu;

constexpr int kCaps[3] = {32, 64, 128};

template <bool WRITE>
int run_cap(int cap, int n, const int *rows, int nrows, const CsrD &A, const CsrD &At, const Params &P, const Out &o,
            cudaStream_t st) {
    if (cap == 32) return launch_rows<32, WRITE>(n, rows, nrows, A, At, P, o, st);
    if (cap == 64) return launch_rows<64, WRITE>(n, rows, nrows, A, At, P, o, st);
    return launch_rows<128, WRITE>(n, rows, nrows, A, At, P, o, st);
}

int build_gpu(int n, const int *Ai, const int *Aj, const double *Av, const Params &P, BuiltGpu &out) {
    FIIM_TRY(check_device(nullptr));
    const long nnz = Ai[n];
    // A^T by counting sort (columns ascend within each row), as the host construction.
    std::vector<int> tp(n + 1, 0), tc(std::max<long>(nnz, 1));
    std::vector<double> tv(std::max<long>(nnz, 1));
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
    cudaStream_t st = nullptr;
    FIIM_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    } guard{st};
    DevBuf mem;
    int *dAi = mem.get<int>(n + 1), *dAj = mem.get<int>(nnz), *dTi = mem.get<int>(n + 1), *dTj = mem.get<int>(nnz);
    double *dAv = mem.get<double>(nnz), *dTv = mem.get<double>(nnz), *dD = mem.get<double>(n);
    int *gcnt = mem.get<int>(n), *hcnt = mem.get<int>(n), *ovf = mem.get<int>(n), *novf = mem.get<int>(1);
    long *goff = mem.get<long>(n), *hoff = mem.get<long>(n);
    int *rows2 = mem.get<int>(n);
    if (!dAi || !dAj || !dTi || !dTj || !dAv || !dTv || !dD || !gcnt || !hcnt || !ovf || !novf || !goff || !hoff ||
        !rows2)
        return set_error(FIIM_ENOMEM, "device allocation for the factor construction failed");
    FIIM_CUDA(cudaMemcpyAsync(dAi, Ai, sizeof(int) * (n + 1), cudaMemcpyHostToDevice, st));
    FIIM_CUDA(cudaMemcpyAsync(dAj, Aj, sizeof(int) * nnz, cudaMemcpyHostToDevice, st));
    FIIM_CUDA(cudaMemcpyAsync(dAv, Av, sizeof(double) * nnz, cudaMemcpyHostToDevice, st));
    FIIM_CUDA(cudaMemcpyAsync(dTi, tp.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, st));
    FIIM_CUDA(cudaMemcpyAsync(dTj, tc.data(), sizeof(int) * nnz, cudaMemcpyHostToDevice, st));
    FIIM_CUDA(cudaMemcpyAsync(dTv, tv.data(), sizeof(double) * nnz, cudaMemcpyHostToDevice, st));
    const CsrD A{dAi, dAj, dAv}, At{dTi, dTj, dTv};
    Out o{gcnt, hcnt, dD, goff, hoff, nullptr, nullptr, nullptr, nullptr, ovf, novf};
    // Pass 1: counts; rows that outgrow a CAP are run again at the next one.
    std::vector<std::vector<int>> pending(3);   // rows each larger CAP serves
    {
        const int *rows = nullptr;
        int nrows = n - 1;
        std::vector<int> h_rows;
        for (int c = 0; c < 3 && n > 1; ++c) {
            FIIM_CUDA(cudaMemsetAsync(novf, 0, sizeof(int), st));
            FIIM_TRY(run_cap<false>(kCaps[c], n, rows, nrows, A, At, P, o, st));
            int no = 0;
            FIIM_CUDA(cudaMemcpyAsync(&no, novf, sizeof(int), cudaMemcpyDeviceToHost, st));
            FIIM_CUDA(cudaStreamSynchronize(st));
            if (c > 0) pending[c] = h_rows;
            if (no == 0) break;
            h_rows.resize(no);
            FIIM_CUDA(cudaMemcpy(h_rows.data(), ovf, sizeof(int) * no, cudaMemcpyDeviceToHost));
            std::sort(h_rows.begin(), h_rows.end());
            if (c == 2)
                return set_error(FIIM_EARG, "row %d's pattern outgrows %d members; use the host construction "
                                            "(fiim_pdfiim_build) or a warpsize cap", h_rows[0], kCaps[2]);
            FIIM_CUDA(cudaMemcpy(rows2, h_rows.data(), sizeof(int) * no, cudaMemcpyHostToDevice));
            rows = rows2;
            nrows = no;
        }
    }
    // Offsets on the host; row 0 is the unit row with D = 1 / (first stored entry of row 0).
    std::vector<int> hg(n, 1), hh(n, 1);
    if (n > 1) {
        FIIM_CUDA(cudaMemcpy(hg.data() + 1, gcnt + 1, sizeof(int) * (n - 1), cudaMemcpyDeviceToHost));
        FIIM_CUDA(cudaMemcpy(hh.data() + 1, hcnt + 1, sizeof(int) * (n - 1), cudaMemcpyDeviceToHost));
    }
    std::vector<long> go(n), ho(n);
    long tg = 0, th = 0;
    for (int i = 0; i < n; ++i) {
        go[i] = tg;
        ho[i] = th;
        tg += hg[i];
        th += hh[i];
    }
    if (tg > 0x7fffffffL || th > 0x7fffffffL) return set_error(FIIM_EARG, "factors too large for int32 CSR");
    int *dgj = mem.get<int>(tg), *dhj = mem.get<int>(th);
    double *dgv = mem.get<double>(tg), *dhv = mem.get<double>(th);
    if (!dgj || !dhj || !dgv || !dhv) return set_error(FIIM_ENOMEM, "device allocation for the factors failed");
    FIIM_CUDA(cudaMemcpyAsync(goff, go.data(), sizeof(long) * n, cudaMemcpyHostToDevice, st));
    FIIM_CUDA(cudaMemcpyAsync(hoff, ho.data(), sizeof(long) * n, cudaMemcpyHostToDevice, st));
    o.gj = dgj;
    o.hj = dhj;
    o.gv = dgv;
    o.hv = dhv;
    // Pass 2: write, every row at the CAP that served it (a row over a CAP skips there).
    if (n > 1) {
        FIIM_TRY(run_cap<true>(kCaps[0], n, nullptr, n - 1, A, At, P, o, st));
        for (int c = 1; c < 3; ++c)
            if (!pending[c].empty()) {
                FIIM_CUDA(cudaMemcpyAsync(rows2, pending[c].data(), sizeof(int) * pending[c].size(),
                                          cudaMemcpyHostToDevice, st));
                FIIM_TRY(run_cap<true>(kCaps[c], n, rows2, (int)pending[c].size(), A, At, P, o, st));
                FIIM_CUDA(cudaStreamSynchronize(st));
            }
    }
    std::vector<int> gj(tg), hj(th);
    std::vector<double> gv(tg), hv(th);
    out.D.resize(n);
    FIIM_CUDA(cudaMemcpyAsync(gj.data(), dgj, sizeof(int) * tg, cudaMemcpyDeviceToHost, st));
    FIIM_CUDA(cudaMemcpyAsync(gv.data(), dgv, sizeof(double) * tg, cudaMemcpyDeviceToHost, st));
    FIIM_CUDA(cudaMemcpyAsync(hj.data(), dhj, sizeof(int) * th, cudaMemcpyDeviceToHost, st));
    FIIM_CUDA(cudaMemcpyAsync(hv.data(), dhv, sizeof(double) * th, cudaMemcpyDeviceToHost, st));
    FIIM_CUDA(cudaMemcpyAsync(out.D.data(), dD, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    FIIM_CUDA(cudaStreamSynchronize(st));
    gj[go[0]] = 0;
    gv[go[0]] = 1.0;
    hj[ho[0]] = 0;
    hv[ho[0]] = 1.0;
    out.D[0] = 1.0 / Av[0];
    // G: column i holds rows gj of row task i; assemble row-wise CSR (ascending i per row).
    out.n = n;
    out.Gi.assign(n + 1, 0);
    for (long q = 0; q < tg; ++q) out.Gi[gj[q] + 1]++;
    for (int r = 0; r < n; ++r) out.Gi[r + 1] += out.Gi[r];
    out.Gj.resize(tg);
    out.Gv.resize(tg);
    {
        std::vector<int> pos(out.Gi.begin(), out.Gi.end() - 1);
        for (int i = 0; i < n; ++i)
            for (long q = go[i]; q < go[i] + hg[i]; ++q) {
                const int at = pos[gj[q]]++;
                out.Gj[at] = i;
                out.Gv[at] = gv[q];
            }
    }
    out.Hi.assign(n + 1, 0);
    for (int i = 0; i < n; ++i) out.Hi[i + 1] = out.Hi[i] + hh[i];
    out.Hj.swap(hj);
    out.Hv.swap(hv);
    return FIIM_OK;
}

}  // namespace pg
}  // namespace fiim

extern "C" int fiim_pdfiim_build_gpu(int n, const int *Ai, const int *Aj, const double *Av, int prefill, int lfill,
                                     int postfill, double ftol, int warpsize, char filttype, char patt, int *nnzG,
                                     int *nnzH, double *Gv, int *Gj, int *Gi, double *D, double *Hv, int *Hj,
                                     int *Hi) {
    using fiim::pg::g_built_gpu;
    if (!Gv) {
        if (n <= 0 || !Ai || !Aj || !Av || !nnzG || !nnzH) return fiim::set_error(FIIM_EARG, "null argument or n <= 0");
        if (patt != 'B') return fiim::set_error(FIIM_EARG, "only the two-sided pattern 'B' is served");
        if (warpsize == 0 || warpsize < -1) return fiim::set_error(FIIM_EARG, "warpsize is -1 or positive");
        g_built_gpu = fiim::pg::BuiltGpu();
        const fiim::pg::Params P{prefill, lfill, postfill, warpsize, ftol, filttype};
        const int rc = fiim::pg::build_gpu(n, Ai, Aj, Av, P, g_built_gpu);
        if (rc != FIIM_OK) {
            g_built_gpu = fiim::pg::BuiltGpu();
            return rc;
        }
        *nnzG = g_built_gpu.Gi[n];
        *nnzH = g_built_gpu.Hi[n];
        return FIIM_OK;
    }
    if (g_built_gpu.n != n || !Gj || !Gi || !D || !Hv || !Hj || !Hi)
        return fiim::set_error(FIIM_EARG, "call first with Gv == NULL, then with every output");
    std::memcpy(Gi, g_built_gpu.Gi.data(), sizeof(int) * (n + 1));
    std::memcpy(Gj, g_built_gpu.Gj.data(), sizeof(int) * g_built_gpu.Gj.size());
    std::memcpy(Gv, g_built_gpu.Gv.data(), sizeof(double) * g_built_gpu.Gv.size());
    std::memcpy(Hi, g_built_gpu.Hi.data(), sizeof(int) * (n + 1));
    std::memcpy(Hj, g_built_gpu.Hj.data(), sizeof(int) * g_built_gpu.Hj.size());
    std::memcpy(Hv, g_built_gpu.Hv.data(), sizeof(double) * g_built_gpu.Hv.size());
    std::memcpy(D, g_built_gpu.D.data(), sizeof(double) * n);
    g_built_gpu = fiim::pg::BuiltGpu();
    return FIIM_OK;
}
