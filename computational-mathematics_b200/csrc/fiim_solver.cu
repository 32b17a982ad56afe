// Host side of the B200 solve phase: device layout, SpMV shape selection, the
// device-driven iteration graph and the handle API of include/fiim_b200.h.
//
// Data layout in HBM (one solver, one arena allocation, 256-byte aligned pieces):
//   A, G, H (L, U for ACIFIM mode 'C'): CSR with int32 row offsets and columns and
//   FP64 values; for a symmetric PDFIIM input, A is expanded to full CSR and
//   H = G^T is formed once at set-up (a gather-form CSR, no atomics in the solve).
//   Vectors x, b, r, r0, p, v, s, t, pc, sc, tm (+ t1, t2, t3 for mode 'C'): FP64[n].
//   DState (device scalars) and per-block reduction partials: a few KB.
//   Mixed precision adds FP32 copies of A, G, H, D^{-1} and FP32 inner vectors.
//
// The solve is three launches: the fused start kernel (r = b - A x, r0, p, ||r0||),
// one CUDA graph whose WHILE node runs the nine-kernel iteration body until the
// device sets its condition to 0, and the FP64 true-residual kernel.

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <iostream>
#include <map>
#include <mutex>
#include <tuple>
#include <string>
#include <vector>

#include "fiim_b200.h"
#include "fiim_internal.h"
#include "fiim_kernels.cuh"
#include "fiim_pipe.cuh"
#include "fiim_persist.cuh"
#include "fiim_cluster.cuh"
#include "fiim_solver.h"

namespace fiim {

// ------------------------------------------------------------------ errors / device
static thread_local std::string g_err;

int set_error(int code, const char *fmt, ...) {
    char buf[768];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

const char *last_error() { return g_err.c_str(); }

int check_device(int *dev_out) {
    int dev = 0, count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return set_error(FIIM_ENODEV, "no CUDA device visible");
    }
    FIIM_CUDA(cudaGetDevice(&dev));
    int major = 0;
    FIIM_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
    if (major != 10)
        return set_error(FIIM_ENODEV, "device %d has compute capability %d.x; this library is built for sm_100a",
                         dev, major);
    if (dev_out) *dev_out = dev;
    return FIIM_OK;
}

int num_sms() {
    static int sms[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (!sms[dev]) cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev);
    return sms[dev] > 0 ? sms[dev] : 148;
}

// ------------------------------------------------------------------ arena
int Arena::reserve(size_t bytes) {
    used = 0;
    if (bytes <= cap) return FIIM_OK;
    release();
    if (cudaMalloc(&base, bytes) != cudaSuccess) {
        cudaGetLastError();
        base = nullptr;
        return set_error(FIIM_ENOMEM, "cudaMalloc of %zu bytes failed", bytes);
    }
    cap = bytes;
    return FIIM_OK;
}

void *Arena::take(size_t bytes) {
    const size_t a = (used + 255) & ~size_t(255);
    if (a + bytes > cap) return nullptr;
    used = a + bytes;
    return static_cast<char *>(base) + a;
}

void Arena::release() {
    if (base) cudaFree(base);
    base = nullptr;
    cap = used = 0;
}

size_t Arena::need(size_t bytes) { return (bytes + 255) & ~size_t(255); }

// ------------------------------------------------------------------ launch shapes
template <int VEC, int FILL, typename Epi>
static cudaError_t spmv_vec(cudaStream_t s, const CsrView<double> &M, const double *x, const Epi &epi,
                            DState *st, double *partials) {
    auto kern = k_spmv_vec<VEC, Epi, FILL>;
    const int g = grid_for(kern, (32 / VEC) * kWarps, M.n);
    kern<<<g, kThreads, 0, s>>>(M, x, epi, st, partials);
    return cudaGetLastError();
}

// Set-up-free SpMV (kernel-level C-ABI): VEC lanes per row, exact row order.
template <int FILL = 0, typename Epi>
cudaError_t launch_spmv_vec(int vec, cudaStream_t s, const CsrView<double> &M, const double *x,
                            const Epi &epi, DState *st, double *partials) {
    switch (vec) {
        case 2: return spmv_vec<2, FILL>(s, M, x, epi, st, partials);
        case 4: return spmv_vec<4, FILL>(s, M, x, epi, st, partials);
        case 8: return spmv_vec<8, FILL>(s, M, x, epi, st, partials);
        case 16: return spmv_vec<16, FILL>(s, M, x, epi, st, partials);
        default: return spmv_vec<32, FILL>(s, M, x, epi, st, partials);
    }
}

static CsrView<double> view(const DevCsr &M) { return CsrView<double>{M.rp, M.ci, M.v, (int)M.n}; }

template <int TILE, typename Epi>
static cudaError_t spmv_rows(cudaStream_t s, const DevCsr &M, const double *x, const Epi &epi,
                             DState *st, double *partials) {
    if (M.narrow) {
        auto kern = k_spmv_rows<TILE, Epi, true>;
        const int g = grid_for(kern, 1, M.nblk);
        return launch_k(kern, g, 0, s, view(M), M.rb, M.eb, M.nblk, x, epi, st, partials, NarrowCols{M.cd, M.cb});
    }
    auto kern = k_spmv_rows<TILE, Epi, false>;
    const int g = grid_for(kern, 1, M.nblk);
    return launch_k(kern, g, 0, s, view(M), M.rb, M.eb, M.nblk, x, epi, st, partials, NarrowCols{});
}

// Resident CTAs per SM of a kernel with `smem` bytes of dynamic shared memory, with the
// attribute that allows it set once per kernel and device.
template <typename K>
static int smem_occupancy(K kern, int smem, int *occ) {
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, int> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(mu);
    const auto key = std::make_pair((const void *)kern, dev);
    auto it = cache.find(key);
    if (it != cache.end()) {
        *occ = it->second;
        return FIIM_OK;
    }
    FIIM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    int b = 0;
    FIIM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, kThreads, smem));
    *occ = cache[key] = std::max(b, 1);
    return FIIM_OK;
}

template <int TILE, typename Epi>
static cudaError_t spmv_pipe(cudaStream_t s, const DevCsr &M, const double *x, const Epi &epi, DState *st,
                             double *partials, int *fault) {
    auto kern = k_spmv_pipe<TILE, Epi>;
    constexpr int smem = PipeSmem<TILE>::kBytes;
    int occ = 1;
    if (smem_occupancy(kern, smem, &occ) != FIIM_OK) return cudaErrorInvalidConfiguration;
    const int g = (int)std::min<long>(std::max(M.nblk, 1), (long)occ * num_sms());
    return launch_k(kern, g, smem, s, view(M), M.rb, M.nblk, x, epi, st, partials, fault);
}

// Warp-block size of the kFormWarp CSR-stream (entries per warp block, 8 per lane).
constexpr int kWarpTile = 256;

template <typename Epi>
static cudaError_t spmv_warp(cudaStream_t s, const DevCsr &M, const double *x, const Epi &epi, DState *st,
                             double *partials) {
    if (M.narrow) {
        auto kern = k_spmv_warp<kWarpTile, Epi, true>;
        const int g = grid_for(kern, kWarps, M.nblk);
        return launch_k(kern, g, 0, s, view(M), M.rb, M.eb, M.nblk, x, epi, st, partials, NarrowCols{M.cd, M.cb});
    }
    auto kern = k_spmv_warp<kWarpTile, Epi, false>;
    const int g = grid_for(kern, kWarps, M.nblk);
    return launch_k(kern, g, 0, s, view(M), M.rb, M.eb, M.nblk, x, epi, st, partials, NarrowCols{});
}

// Sliced-diagonal SpMV: kWarps warps per CTA, one slice per warp trip.
template <typename Epi>
static cudaError_t spmv_dia(cudaStream_t s, const DevCsr &M, const double *x, const Epi &epi, DState *st,
                            double *partials) {
    if (M.dseg) return cudaErrorInvalidValue;   // k_spmv_dia takes slices of one segment
    const DiaView<double> view{M.drec, static_cast<const double *>(M.dvals), (int)M.n, M.nsl, M.drs};
    if (M.dsh == 64) {
        auto kern = k_spmv_dia<double, double, 2, Epi>;
        return launch_k(kern, grid_for(kern, kWarps, M.nsl), 0, s, view, x, epi, st, partials);
    }
    auto kern = k_spmv_dia<double, double, 1, Epi>;
    return launch_k(kern, grid_for(kern, kWarps, M.nsl), 0, s, view, x, epi, st, partials);
}

// Solver SpMV: the sliced-diagonal copy where the matrix has one, else CSR-stream over the
// matrix's row blocks, in the form and row-block size the tuner chose. Every form gives the
// same bits.
template <typename Epi>
cudaError_t launch_spmv(const DevCsr &M, cudaStream_t s, const double *x, const Epi &epi, DState *st,
                        double *partials, int *fault = nullptr) {
    if (M.dia) return spmv_dia(s, M, x, epi, st, partials);
    if (M.form == kFormWarp) return spmv_warp(s, M, x, epi, st, partials);
    if (M.form == kFormBulk && fault) {
        if (M.tile == 1024) return spmv_pipe<1024>(s, M, x, epi, st, partials, fault);
        return spmv_pipe<2048>(s, M, x, epi, st, partials, fault);
    }
    switch (M.tile) {
        case 512: return spmv_rows<512>(s, M, x, epi, st, partials);
        case 1024: return spmv_rows<1024>(s, M, x, epi, st, partials);
        case 4096: return spmv_rows<4096>(s, M, x, epi, st, partials);
        default: return spmv_rows<2048>(s, M, x, epi, st, partials);
    }
}

template <typename K>
static int stream_grid(K kernel, long n) { return grid_for(kernel, kThreads, n); }

int heuristic_vec(long n, long nnz) {
    const double mean = n > 0 ? (double)nnz / (double)n : 1.0;
    int v = 2;
    while (v < 32 && v < mean) v <<= 1;
    return v;
}

void build_row_blocks(const std::vector<int> &rp, int tile, int max_rows, std::vector<int> &rb) {
    const int n = (int)rp.size() - 1;
    rb.clear();
    rb.push_back(0);
    int r = 0;
    while (r < n) {
        if (rp[r + 1] - rp[r] > tile) {
            rb.push_back(++r);
            continue;
        }
        const int start = r;
        long nnz = 0;
        while (r < n && r - start < max_rows && nnz + (rp[r + 1] - rp[r]) <= tile) {
            nnz += rp[r + 1] - rp[r];
            ++r;
        }
        rb.push_back(r);
    }
}

int build_narrow(DevCsr &M, cudaStream_t s) {
    // Narrow column stream when every row block allows it (FIIM_COLS=wide keeps 32-bit columns).
    M.narrow = 0;
    const char *cols = std::getenv("FIIM_COLS");
    if (M.nblk > 0 && M.nnz > 0 && M.cd && !(cols && std::strcmp(cols, "wide") == 0)) {
        FIIM_CUDA(cudaMemsetAsync(M.wide, 0, sizeof(int), s));
        const int g = (int)std::min<long>(M.nblk, 16L * num_sms());
        k_narrow_cols<<<g, kThreads, 0, s>>>(M.ci, M.eb, M.nblk, M.cd, M.cb, M.wide);
        FIIM_CUDA(cudaGetLastError());
        int wide = 1;
        FIIM_CUDA(cudaMemcpyAsync(&wide, M.wide, sizeof(int), cudaMemcpyDeviceToHost, s));
        FIIM_CUDA(cudaStreamSynchronize(s));
        M.narrow = wide ? 0 : 1;
    }
    return FIIM_OK;
}

void release_dia(DevCsr &M) {
    if (M.dia_mem) cudaFree(M.dia_mem);
    M.dia_mem = nullptr;
    M.dia_bytes = 0;
    M.drec = M.dmap = M.dbad = nullptr;
    M.dvals = nullptr;
    M.dvbytes = 0;
    M.dsh = 0;
    M.dseg = false;
    M.dia = 0;
    M.nsl = 0;
    M.drs = 0;
    M.ndiag = 0;
}

bool dia_wanted() {
    // FIIM_SPMV=rows / staged / warp keep a CSR-stream form; FIIM_DIA=0 never builds the copy.
    const char *force = std::getenv("FIIM_SPMV"), *off_env = std::getenv("FIIM_DIA");
    return !((force && std::strcmp(force, "dia") != 0) || (off_env && std::strcmp(off_env, "0") == 0));
}

template <typename B>
static int place_bits(DevCsr &M, const void *vals, B pad, cudaStream_t s) {
    const long slots = (long)M.dsh * M.ndiag;
    B *dv = static_cast<B *>(M.dvals);
    k_dia_fill<B><<<stream_grid(k_dia_fill<B>, slots), kThreads, 0, s>>>(slots, dv, pad);
    FIIM_CUDA(cudaGetLastError());
    k_dia_scatter<B><<<stream_grid(k_dia_scatter<B>, M.nnz), kThreads, 0, s>>>(M.nnz, static_cast<const B *>(vals),
                                                                               M.dmap, dv, pad, M.dbad);
    FIIM_CUDA(cudaGetLastError());
    return FIIM_OK;
}

int place_dia(DevCsr &M, const void *vals, cudaStream_t s) {
    if (!M.dia_mem) return FIIM_OK;
    FIIM_CUDA(cudaMemsetAsync(M.dbad, 0, sizeof(int), s));
    if (M.dvbytes == 8) FIIM_TRY(place_bits<unsigned long long>(M, vals, kDiaPad, s));
    else if (M.dvbytes == 4) FIIM_TRY(place_bits<unsigned>(M, vals, kDiaPad32, s));
    else FIIM_TRY(place_bits<unsigned short>(M, vals, kDiaPad16, s));
    int bad = 0;
    FIIM_CUDA(cudaMemcpyAsync(&bad, M.dbad, sizeof(int), cudaMemcpyDeviceToHost, s));
    FIIM_CUDA(cudaStreamSynchronize(s));
    if (bad) release_dia(M);   // an entry holds the padding pattern: the CSR streams serve
    else M.dia = 1;
    return FIIM_OK;
}

static int col_hash(DevCsr &M, cudaStream_t s, unsigned long long *h) {
    *h = 0;
    if (M.nnz <= 0 || !M.dhash) return FIIM_OK;
    FIIM_CUDA(cudaMemsetAsync(M.dhash, 0, sizeof(unsigned long long), s));
    k_col_hash<<<stream_grid(k_col_hash, M.nnz), kThreads, 0, s>>>(M.nnz, M.ci, M.dhash);
    FIIM_CUDA(cudaGetLastError());
    FIIM_CUDA(cudaMemcpyAsync(h, M.dhash, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    FIIM_CUDA(cudaStreamSynchronize(s));
    return FIIM_OK;
}

int dia_rows_per_lane(int vbytes) {
    if (vbytes == 8) {
        const char *e = std::getenv("FIIM_DIA_R");
        return (e && (e[0] == '1' || e[0] == '2') && e[1] == 0) ? e[0] - '0' : 0;   // 0: by the matrix
    }
    return vbytes == 4 ? 2 : 4;
}

int build_dia_structure(DevCsr &M, cudaStream_t s, int vbytes, const std::vector<int> *segments) {
    release_dia(M);
    M.dia_tried = false;
    M.hseg_sl.clear();
    if (!dia_wanted()) return FIIM_OK;
    const int n = (int)M.n;
    const long nnz = M.nnz;
    if (n <= 0 || nnz <= 0 || (long)M.hrp.size() != (long)n + 1) return FIIM_OK;
    const std::vector<int> whole = {0, n};
    const std::vector<int> &seg = segments ? *segments : whole;
    if (seg.size() < 2 || seg.front() != 0 || seg.back() != n) return set_error(FIIM_EARG, "segments must cover the rows");
    FIIM_TRY(col_hash(M, s, &M.dia_cols));
    M.dia_tried = true;
    std::vector<int> ci(nnz);
    FIIM_CUDA(cudaMemcpyAsync(ci.data(), M.ci, sizeof(int) * nnz, cudaMemcpyDeviceToHost, s));
    FIIM_CUDA(cudaStreamSynchronize(s));
    const int *rp = M.hrp.data();
    // Slices of up to sh rows, never straddling a segment: first row, rows, and each segment's
    // first slice.
    int sh = 0, nsl = 0;
    std::vector<int> first, rows, seg_sl;
    auto slices = [&](int R) {
        sh = 32 * R;
        first.clear();
        rows.clear();
        seg_sl.assign(1, 0);
        for (size_t q = 0; q + 1 < seg.size(); ++q) {
            for (int r = seg[q]; r < seg[q + 1]; r += sh) {
                first.push_back(r);
                rows.push_back(std::min(sh, seg[q + 1] - r));
            }
            seg_sl.push_back((int)first.size());
        }
        nsl = (int)first.size();
    };
    // The diagonals of a slice: its entries' col - row, sorted and distinct.
    auto diagonals = [&](int sl, std::vector<int> &d, int &unsorted) {
        d.clear();
        const int r0 = first[sl], r1 = r0 + rows[sl];
        for (int i = r0; i < r1; ++i)
            for (int e = rp[i]; e < rp[i + 1]; ++e) {
                if (e > rp[i] && ci[e] <= ci[e - 1]) unsorted = 1;
                d.push_back(ci[e] - i);
            }
        std::sort(d.begin(), d.end());
        d.erase(std::unique(d.begin(), d.end()), d.end());
    };
    // Diagonals per slice for R rows a lane (sp[sl + 1]); false when a row is unsorted or a
    // slice has more than kDiaMaxDiags.
    std::vector<int> sp;
    auto count = [&](int R) -> bool {
        slices(R);
        sp.assign(nsl + 1, 0);
        std::atomic<int> fail{0};   // a failed slice ends the analysis (random matrices fail at once)
#pragma omp parallel
        {
            std::vector<int> d;
#pragma omp for schedule(dynamic, 256)
            for (int sl = 0; sl < nsl; ++sl) {
                if (fail.load(std::memory_order_relaxed)) continue;
                int bad = 0;
                diagonals(sl, d, bad);
                sp[sl + 1] = (int)d.size();
                if (bad || (int)d.size() > kDiaMaxDiags) fail.store(1, std::memory_order_relaxed);
            }
        }
        return !fail.load();
    };
    // FP64 takes two rows a lane when its 32-row slices average more diagonals than one chunk
    // of the kernel holds (H at 128^3: 11 diagonals, 32.9 against 41.6 us a product; A and G,
    // 7 diagonals, were slower with two).
    int R = dia_rows_per_lane(vbytes);
    if (R == 0) {
        if (!count(1)) return FIIM_OK;
        long nd1 = 0;
        for (int sl = 0; sl < nsl; ++sl) nd1 += sp[sl + 1];
        R = 1;
        if (nd1 > 8L * nsl) {
            if (count(2)) R = 2;
            else if (!count(1)) return FIIM_OK;
        }
    } else if (!count(R)) {
        return FIIM_OK;
    }
    int most = 0;
    for (int sl = 0; sl < nsl; ++sl) {
        most = std::max(most, sp[sl + 1]);
        sp[sl + 1] += sp[sl];
    }
    const long ndiag = sp[nsl];
    const int rs = most <= 16 - kDiaRecHead - 2 ? 16 : 32;
    // Kept only when it moves fewer bytes than the CSR streams it replaces.
    const double dia_bytes = (double)vbytes * sh * ndiag + 4.0 * rs * nsl;
    const double csr_bytes_now = (double)nnz * (vbytes + (M.narrow ? 2 : 4)) + 4.0 * (n + 1);
    if (!(dia_bytes < csr_bytes_now) || (long)sh * ndiag >= (1L << 31)) return FIIM_OK;
    std::vector<int> rec((size_t)nsl * rs, 0), map(nnz);
#pragma omp parallel
    {
        std::vector<int> d;
        int unused = 0;
#pragma omp for schedule(dynamic, 256)
        for (int sl = 0; sl < nsl; ++sl) {
            diagonals(sl, d, unused);
            int *r = rec.data() + (size_t)sl * rs;
            const int r0 = first[sl], r1 = r0 + rows[sl];
            // Every slot of the slice (rows r0 .. r0 + sh - 1, padding included) gathers a column
            // r + d: the slice is flagged when one of them falls outside [0, n).
            const bool outside = !d.empty() && ((long)r0 + d.front() < 0 || (long)r0 + sh - 1 + d.back() > n - 1);
            r[0] = sp[sl];
            r[1] = (int)d.size() | (outside ? kDiaClamp : 0);
            r[rs - 2] = r0;
            r[rs - 1] = rows[sl];
            std::copy(d.begin(), d.end(), r + kDiaRecHead);
            for (int i = r0; i < r1; ++i)
                for (int e = rp[i]; e < rp[i + 1]; ++e) {
                    const int k = (int)(std::lower_bound(d.begin(), d.end(), ci[e] - i) - d.begin());
                    map[e] = sh * (sp[sl] + k) + (i - r0);
                }
        }
    }
    const size_t b_rec = Arena::need(sizeof(int) * rec.size()), b_map = Arena::need(sizeof(int) * nnz),
                 b_bad = Arena::need(sizeof(int)), b_v = Arena::need((size_t)vbytes * sh * ndiag);
    char *mem = nullptr;
    if (cudaMalloc(&mem, b_rec + b_map + b_bad + b_v) != cudaSuccess) {
        cudaGetLastError();
        return FIIM_OK;   // no room for the copy: the CSR streams serve
    }
    M.dia_mem = mem;
    M.dia_bytes = b_rec + b_map + b_bad + b_v;
    M.drec = reinterpret_cast<int *>(mem);
    M.dmap = reinterpret_cast<int *>(mem + b_rec);
    M.dbad = reinterpret_cast<int *>(mem + b_rec + b_map);
    M.dvals = mem + b_rec + b_map + b_bad;
    M.dvbytes = vbytes;
    M.dsh = sh;
    M.nsl = nsl;
    M.drs = rs;
    M.ndiag = ndiag;
    M.hseg_sl = seg_sl;
    M.dseg = seg.size() > 2;
    FIIM_CUDA(cudaMemcpyAsync(M.drec, rec.data(), sizeof(int) * rec.size(), cudaMemcpyHostToDevice, s));
    FIIM_CUDA(cudaMemcpyAsync(M.dmap, map.data(), sizeof(int) * nnz, cudaMemcpyHostToDevice, s));
    FIIM_CUDA(cudaStreamSynchronize(s));   // before the host arrays go
    return FIIM_OK;
}

int dia_fits(DevCsr &M, cudaStream_t s, bool *fits) {
    *fits = false;
    if (!M.dia_mem) return FIIM_OK;
    FIIM_CUDA(cudaMemsetAsync(M.dbad, 0, sizeof(int), s));
    const int g = (int)std::min<long>((M.nsl + kWarps - 1) / kWarps, 16L * num_sms());
    k_dia_check<<<std::max(g, 1), kThreads, 0, s>>>(M.nsl, M.rp, M.ci, M.dmap, M.drec, M.drs, M.dsh, M.dbad);
    FIIM_CUDA(cudaGetLastError());
    int bad = 0;
    FIIM_CUDA(cudaMemcpyAsync(&bad, M.dbad, sizeof(int), cudaMemcpyDeviceToHost, s));
    FIIM_CUDA(cudaStreamSynchronize(s));
    *fits = !bad;
    return FIIM_OK;
}

int build_dia(DevCsr &M, cudaStream_t s) {
    FIIM_TRY(build_dia_structure(M, s, 8));
    return place_dia(M, M.v, s);
}

int refresh_dia(DevCsr &M, cudaStream_t s) {
    if (!dia_wanted()) return FIIM_OK;
    if (!M.dia) {   // not built for the previous columns: decide again only if they changed
        unsigned long long h = 0;
        FIIM_TRY(col_hash(M, s, &h));
        if (M.dia_tried && h == M.dia_cols) return FIIM_OK;
        return build_dia(M, s);
    }
    bool fits = false;
    FIIM_TRY(dia_fits(M, s, &fits));
    if (!fits) return build_dia(M, s);
    return place_dia(M, M.v, s);
}

// refresh_dia for a copy whose row offsets did not change, enqueued on `aux` once the copies
// of M's columns and values (issued on `copy_s` before this call) are done, so it runs while
// later copies do. The columns fit only when they equal those the copy was built for (the
// check holds each entry to its slot), so the padding slots stay as they were and need no
// fill; the check and the value scatter share M.dbad, which lands in *h_bad (pinned). 0 there
// after `aux` synchronizes: the copy holds the new values. Otherwise the values in the copy
// are not to be used, and refresh_dia decides again.
static int refresh_dia_async(DevCsr &M, cudaStream_t copy_s, cudaStream_t aux, cudaEvent_t done, int *h_bad) {
    FIIM_CUDA(cudaEventRecord(done, copy_s));
    FIIM_CUDA(cudaStreamWaitEvent(aux, done, 0));
    FIIM_CUDA(cudaMemsetAsync(M.dbad, 0, sizeof(int), aux));
    const int g = (int)std::min<long>((M.nsl + kWarps - 1) / kWarps, 16L * num_sms());
    k_dia_check<<<std::max(g, 1), kThreads, 0, aux>>>(M.nsl, M.rp, M.ci, M.dmap, M.drec, M.drs, M.dsh, M.dbad);
    FIIM_CUDA(cudaGetLastError());
    using B = unsigned long long;
    k_dia_scatter<B><<<stream_grid(k_dia_scatter<B>, M.nnz), kThreads, 0, aux>>>(
        M.nnz, reinterpret_cast<const B *>(M.v), M.dmap, static_cast<B *>(M.dvals), kDiaPad, M.dbad);
    FIIM_CUDA(cudaGetLastError());
    FIIM_CUDA(cudaMemcpyAsync(h_bad, M.dbad, sizeof(int), cudaMemcpyDeviceToHost, aux));
    return FIIM_OK;
}

int set_tile(DevCsr &M, int tile, cudaStream_t s) {
    std::vector<int> rb;
    // k_spmv_rows reads aligned pairs (blocks of at most tile - 1 entries); a warp block has
    // at most 32 rows, a CTA block kThreads.
    build_row_blocks(M.hrp, tile - 1, M.form == kFormWarp ? 32 : kThreads, rb);
    M.tile = tile;
    M.nblk = (int)rb.size() - 1;
    std::vector<int> eb(rb.size());
    for (size_t k = 0; k < rb.size(); ++k) eb[k] = M.hrp[rb[k]];
    FIIM_CUDA(cudaMemcpyAsync(M.rb, rb.data(), sizeof(int) * rb.size(), cudaMemcpyHostToDevice, s));
    FIIM_CUDA(cudaMemcpyAsync(M.eb, eb.data(), sizeof(int) * eb.size(), cudaMemcpyHostToDevice, s));
    FIIM_TRY(build_narrow(M, s));
    FIIM_CUDA(cudaStreamSynchronize(s));
    return FIIM_OK;
}

// Row-block size used when timing-based tuning is off. With the row-block loop pipelined
// (next block's stream and epilogue operands in registers), 2048 entries per block was the
// fastest size for the 7-, 6- and 11-entry rows of the 3D convection-diffusion A, G and H.
static int default_tile(const DevCsr &) { return 2048; }

// Largest system the one-launch solve takes (its per-phase work stays a few microseconds).
constexpr int kPersistMaxN = 65536;

// Time each row-block size on this matrix and keep the fastest; cached by signature.
// The choice changes speed only: every shape sums each row in storage order.
static int autotune_tile(DevCsr &M, const double *x, double *y, cudaStream_t s, int *fault) {
    static std::mutex mu;
    static std::map<std::vector<long>, std::pair<int, int>> cache;
    // FIIM_SPMV=rows or FIIM_SPMV=staged restricts the candidates to one form (tests use it
    // to cover both; the results are the same bits in either form).
    const char *force = std::getenv("FIIM_SPMV");
    const int only = !force ? -1
                            : (std::strcmp(force, "rows") == 0     ? kFormRows
                               : std::strcmp(force, "staged") == 0 ? kFormBulk
                               : std::strcmp(force, "warp") == 0   ? kFormWarp
                                                                   : -1);
    std::vector<long> key = M.sig;
    key.push_back(only);
    std::pair<int, int> cached{0, 0};
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find(key);
        if (it != cache.end()) cached = it->second;
    }
    if (cached.first) {
        M.form = cached.second;
        return set_tile(M, cached.first, s);
    }
    // Candidates (row-block size, form).
    const std::pair<int, int> cands[] = {{512, kFormRows},  {1024, kFormRows}, {2048, kFormRows},
                                         {4096, kFormRows},  {1024, kFormBulk}, {2048, kFormBulk},
                                         {kWarpTile, kFormWarp}};
    cudaEvent_t e0, e1;
    FIIM_CUDA(cudaEventCreate(&e0));
    FIIM_CUDA(cudaEventCreate(&e1));
    std::pair<int, int> best{0, 0};
    float best_ms = 1e30f;
    const int reps = M.nnz > 4000000 ? 5 : 10;
    for (const auto &c : cands) {
        if (only >= 0 && c.second != only) continue;
        M.form = c.second;
        FIIM_TRY(set_tile(M, c.first, s));
        FIIM_CUDA(launch_spmv(M, s, x, EpiStore{y}, nullptr, nullptr, fault));
        FIIM_CUDA(cudaEventRecord(e0, s));
        for (int r = 0; r < reps; ++r) FIIM_CUDA(launch_spmv(M, s, x, EpiStore{y}, nullptr, nullptr, fault));
        FIIM_CUDA(cudaEventRecord(e1, s));
        FIIM_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        FIIM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (!best.first || ms < best_ms * 0.97f) {
            best_ms = ms;
            best = c;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    {
        std::lock_guard<std::mutex> lk(mu);
        cache[key] = best;
    }
    M.form = best.second;
    return set_tile(M, best.first, s);
}

// ------------------------------------------------------------------ host CSR helpers
// Full CSR of a symmetric matrix given by its stored upper triangle (entries with
// col < row are ignored, as MKL's SYMMETRIC + UPPER descriptor does).
void expand_sym_upper(int n, const int *rp, const int *ci, const double *v, HostCsr &out) {
    out.n = n;
    out.rp.assign(n + 1, 0);
    for (int i = 0; i < n; ++i)
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            const int j = ci[k];
            if (j < i) continue;
            out.rp[i + 1]++;
            if (j != i) out.rp[j + 1]++;
        }
    for (int i = 0; i < n; ++i) out.rp[i + 1] += out.rp[i];
    out.ci.resize(out.rp[n]);
    out.v.resize(out.rp[n]);
    std::vector<int> pos(out.rp.begin(), out.rp.end() - 1);
    // Mirrored (lower) entries first: row j receives (j, i) for i < j in increasing i,
    // then its own upper entries in stored order, so columns stay ascending.
    std::vector<int> lower_count(n, 0);
    for (int i = 0; i < n; ++i)
        for (int k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] > i) lower_count[ci[k]]++;
    std::vector<int> upos(n);
    for (int i = 0; i < n; ++i) upos[i] = out.rp[i] + lower_count[i];
    for (int i = 0; i < n; ++i)
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            const int j = ci[k];
            if (j < i) continue;
            out.ci[upos[i]] = j;
            out.v[upos[i]++] = v[k];
            if (j != i) {
                out.ci[pos[j]] = i;
                out.v[pos[j]++] = v[k];
            }
        }
}

// CSR of T^T where T is the upper triangle (col >= row) of (rp, ci, v).
void transpose_upper(int n, const int *rp, const int *ci, const double *v, HostCsr &out) {
    out.n = n;
    out.rp.assign(n + 1, 0);
    for (int i = 0; i < n; ++i)
        for (int k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] >= i) out.rp[ci[k] + 1]++;
    for (int i = 0; i < n; ++i) out.rp[i + 1] += out.rp[i];
    out.ci.resize(out.rp[n]);
    out.v.resize(out.rp[n]);
    std::vector<int> pos(out.rp.begin(), out.rp.end() - 1);
    for (int i = 0; i < n; ++i)
        for (int k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] >= i) {
                out.ci[pos[ci[k]]] = i;
                out.v[pos[ci[k]]++] = v[k];
            }
}

void signature(DevCsr &M, const int *host_rp) {
    M.sig.clear();
    M.sig.push_back(M.n);
    M.sig.push_back(M.nnz);
    const long step = std::max<long>(1, M.n / 64);
    for (long i = 0; i <= M.n; i += step) M.sig.push_back(host_rp[i]);
    M.sig.push_back(host_rp[M.n]);
}

// Upload one CSR matrix into pre-carved buffers (capacity nnz_cap), in two halves:
// upload_csr_async issues the copies (the column and value arrays first; a host-side row
// offset array is compared with the previous upload's while they run, and copied only if it
// differs), and check_fill_launch / check_fill_finish apply MKL's TRIANGULAR fill semantics:
// fill 1 keeps col >= row, fill 2 keeps col <= row (AFIIM/src/bicgstab.cpp:140-147). The check
// runs on the device; the rare matrix with entries outside its triangle is compacted on the
// host. A caller uploading several matrices issues every copy and check before one sync.
int Stager::copy(void *dst, const void *src, size_t bytes, cudaStream_t s) {
    cudaPointerAttributes attr{};
    const bool pageable = cudaPointerGetAttributes(&attr, src) == cudaSuccess && attr.type == cudaMemoryTypeUnregistered;
    cudaGetLastError();
    if (!pageable || bytes < kMinStaged) {
        FIIM_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
        return FIIM_OK;
    }
    if (!buf[0]) {
        for (int k = 0; k < kBufs; ++k) {
            if (cudaHostAlloc(&buf[k], kChunk, cudaHostAllocDefault) != cudaSuccess) {
                cudaGetLastError();
                release();
                FIIM_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));   // no pinned memory
                return FIIM_OK;
            }
            FIIM_CUDA(cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming));
        }
    }
    const char *in = static_cast<const char *>(src);
    char *out = static_cast<char *>(dst);
    for (size_t off = 0; off < bytes; off += kChunk) {
        const size_t len = std::min(kChunk, bytes - off);
        const int k = next;
        next = (next + 1) % kBufs;
        if (pending[k]) FIIM_CUDA(cudaEventSynchronize(ev[k]));   // the buffer's previous DMA
        char *pb = static_cast<char *>(buf[k]);
        const long parts = (long)((len + (size_t(1) << 20) - 1) >> 20);
#pragma omp parallel for schedule(static)
        for (long q = 0; q < parts; ++q) {
            const size_t a = (size_t)q << 20, e = std::min(len, a + (size_t(1) << 20));
            std::memcpy(pb + a, in + off + a, e - a);
        }
        FIIM_CUDA(cudaMemcpyAsync(out + off, pb, len, cudaMemcpyHostToDevice, s));
        FIIM_CUDA(cudaEventRecord(ev[k], s));
        pending[k] = true;
    }
    return FIIM_OK;
}

void Stager::release() {
    for (int k = 0; k < kBufs; ++k) {
        if (ev[k]) {
            cudaEventSynchronize(ev[k]);
            cudaEventDestroy(ev[k]);
        }
        if (buf[k]) cudaFreeHost(buf[k]);
        ev[k] = nullptr;
        buf[k] = nullptr;
        pending[k] = false;
    }
    next = 0;
}

int upload_csr_async(DevCsr &M, long nnz_cap, int n, const int *rp, const int *ci, const double *v, bool device_src,
                     cudaStream_t s, Stager *stager) {
    std::vector<int> &hrp = M.hrp;
    const bool had = (M.n == n && (long)hrp.size() == (long)n + 1);
    M.n = n;
    const cudaMemcpyKind kind = device_src ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    if (device_src) {
        std::vector<int> nrp(n + 1);
        FIIM_CUDA(cudaMemcpyAsync(nrp.data(), rp, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, s));
        FIIM_CUDA(cudaStreamSynchronize(s));
        M.rows_same = had && nrp == hrp;
        hrp.swap(nrp);
        const long nnz = hrp[n];
        if (nnz > nnz_cap) return set_error(FIIM_EARG, "matrix has %ld entries, capacity %ld", nnz, nnz_cap);
        if (nnz < 0) return set_error(FIIM_EARG, "negative row offset at n");
        M.nnz = nnz;
        FIIM_CUDA(cudaMemcpyAsync(M.rp, rp, sizeof(int) * (n + 1), kind, s));
        if (nnz > 0) {
            FIIM_CUDA(cudaMemcpyAsync(M.ci, ci, sizeof(int) * nnz, kind, s));
            FIIM_CUDA(cudaMemcpyAsync(M.v, v, sizeof(double) * nnz, kind, s));
        }
    } else {
        const long nnz = rp[n];
        if (nnz > nnz_cap) return set_error(FIIM_EARG, "matrix has %ld entries, capacity %ld", nnz, nnz_cap);
        if (nnz < 0) return set_error(FIIM_EARG, "negative row offset at n");
        M.nnz = nnz;
        auto h2d = [&](void *dst, const void *src, size_t bytes) -> int {
            if (stager) return stager->copy(dst, src, bytes, s);
            FIIM_CUDA(cudaMemcpyAsync(dst, src, bytes, kind, s));
            return FIIM_OK;
        };
        if (nnz > 0) {
            FIIM_TRY(h2d(M.ci, ci, sizeof(int) * nnz));
            FIIM_TRY(h2d(M.v, v, sizeof(double) * nnz));
        }
        // The device keeps the previous upload's offsets (hrp mirrors them): copy only on change.
        M.rows_same = had && std::memcmp(hrp.data(), rp, sizeof(int) * (n + 1)) == 0;
        if (!M.rows_same) {
            hrp.resize(n + 1);
            std::memcpy(hrp.data(), rp, sizeof(int) * (n + 1));
            FIIM_TRY(h2d(M.rp, rp, sizeof(int) * (n + 1)));
        }
    }
    signature(M, hrp.data());
    return FIIM_OK;
}

int check_fill_launch(DevCsr &M, int fill, cudaStream_t s, unsigned long long *d_count, unsigned long long *h_count) {
    *h_count = 0;
    if (fill == 0 || M.nnz == 0) return FIIM_OK;
    FIIM_CUDA(cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), s));
    const int n = (int)M.n;
    const int g = std::min(num_sms() * 8, std::max(1, (n + kThreads - 1) / kThreads));
    k_count_outside<<<g, kThreads, 0, s>>>(n, M.rp, M.ci, fill == 1, d_count);
    FIIM_CUDA(cudaGetLastError());
    FIIM_CUDA(cudaMemcpyAsync(h_count, d_count, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    return FIIM_OK;
}

// After the stream has synchronized: compact M to its triangle if the check found entries
// outside it.
int check_fill_finish(DevCsr &M, int fill, unsigned long long outside) {
    if (fill == 0 || outside == 0) return FIIM_OK;
    const int n = (int)M.n;
    const long nnz = M.nnz;
    std::vector<int> crp(n + 1), cci(nnz);
    std::vector<double> cv(nnz);
    FIIM_CUDA(cudaMemcpy(crp.data(), M.rp, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost));
    FIIM_CUDA(cudaMemcpy(cci.data(), M.ci, sizeof(int) * nnz, cudaMemcpyDeviceToHost));
    FIIM_CUDA(cudaMemcpy(cv.data(), M.v, sizeof(double) * nnz, cudaMemcpyDeviceToHost));
    long c = 0;
    std::vector<int> nrp(n + 1, 0);
    for (int i = 0; i < n; ++i) {
        for (int k = crp[i]; k < crp[i + 1]; ++k) {
            const int j = cci[k];
            if ((fill == 1) ? (j >= i) : (j <= i)) {
                cci[c] = j;
                cv[c] = cv[k];
                ++c;
            }
        }
        nrp[i + 1] = (int)c;
    }
    M.nnz = c;
    FIIM_CUDA(cudaMemcpy(M.rp, nrp.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
    if (c > 0) {
        FIIM_CUDA(cudaMemcpy(M.ci, cci.data(), sizeof(int) * c, cudaMemcpyHostToDevice));
        FIIM_CUDA(cudaMemcpy(M.v, cv.data(), sizeof(double) * c, cudaMemcpyHostToDevice));
    }
    M.hrp.swap(nrp);
    M.rows_same = false;   // the stored offsets are the filtered ones
    signature(M, M.hrp.data());
    return FIIM_OK;
}

int upload_csr(DevCsr &M, long nnz_cap, int n, const int *rp, const int *ci, const double *v, int fill,
               bool device_src, cudaStream_t s, unsigned long long *d_count, unsigned long long *h_count) {
    FIIM_TRY(upload_csr_async(M, nnz_cap, n, rp, ci, v, device_src, s));
    if (fill == 0 || M.nnz == 0) return FIIM_OK;
    FIIM_TRY(check_fill_launch(M, fill, s, d_count, h_count));
    FIIM_CUDA(cudaStreamSynchronize(s));
    return check_fill_finish(M, fill, *h_count);
}

// Uploads of the solver's matrices: every copy and triangle check issued, then one sync.
static int upload_all(DevCsr *const *mats, const long *caps, const int *const *rps, const int *const *cis,
                      const double *const *vs, const int *fills, const bool *dev, int count, int n, cudaStream_t s,
                      unsigned long long *d_count, unsigned long long *h_count, Stager *stager,
                      const std::function<int(int)> &issued = nullptr) {
    for (int k = 0; k < count; ++k) {
        FIIM_TRY(upload_csr_async(*mats[k], caps[k], n, rps[k], cis[k], vs[k], dev[k], s, stager));
        if (issued) FIIM_TRY(issued(k));   // matrix k's copies are on the stream
    }
    for (int k = 0; k < count; ++k) FIIM_TRY(check_fill_launch(*mats[k], fills[k], s, d_count + k, h_count + k));
    FIIM_CUDA(cudaStreamSynchronize(s));
    for (int k = 0; k < count; ++k) FIIM_TRY(check_fill_finish(*mats[k], fills[k], h_count[k]));
    return FIIM_OK;
}

// Column and value arrays get kStreamSlack bytes after their last entry: the staged SpMV
// forms copy 16-byte aligned windows that may end up to 12 bytes past a block's last entry.
constexpr size_t kStreamSlack = 16;

int carve_csr(Arena &ar, DevCsr &M, long n, long nnz) {
    M.rp = static_cast<int *>(ar.take(sizeof(int) * (n + 1)));
    M.ci = static_cast<int *>(ar.take(sizeof(int) * std::max<long>(nnz, 1) + kStreamSlack));
    M.v = static_cast<double *>(ar.take(sizeof(double) * std::max<long>(nnz, 1) + kStreamSlack));
    M.rb = static_cast<int *>(ar.take(sizeof(int) * (3 * (n + 1) + 6)));   // at most one block per row
    M.cd = static_cast<short *>(ar.take(sizeof(short) * std::max<long>(nnz, 1) + kStreamSlack));
    if (!M.rp || !M.ci || !M.v || !M.rb || !M.cd) return set_error(FIIM_ENOMEM, "arena exhausted");
    M.eb = M.rb + (n + 1);
    M.cb = M.rb + 2 * (n + 1);
    M.wide = M.rb + 3 * (n + 1);
    M.dhash = reinterpret_cast<unsigned long long *>(M.rb + ((3 * (n + 1) + 3) & ~1L));   // 8-byte aligned
    return FIIM_OK;
}

size_t csr_bytes(long n, long nnz) {
    return Arena::need(sizeof(int) * (n + 1)) + Arena::need(sizeof(int) * (3 * (n + 1) + 6)) +
           Arena::need(sizeof(short) * std::max<long>(nnz, 1) + kStreamSlack) +
           Arena::need(sizeof(int) * std::max<long>(nnz, 1) + kStreamSlack) +
           Arena::need(sizeof(double) * std::max<long>(nnz, 1) + kStreamSlack);
}

// ------------------------------------------------------------------ preconditioner
// out = M in for the chosen preconditioner; the last product's epilogue stores the
// result and, when `norm`, also accumulates ||out||^2 into st->pc2.
int Solver::enqueue_prec(const double *in, double *out, bool norm) {
    cudaStream_t s = stream;
    const bool combined = (opt.variant == FIIM_ACIFIM && opt.mode == 'C' && opt.nr > 1);
    if (!combined) {
        // tm = IDv o (H in); out = G tm   (AFIIM/src/bicgstab.cpp:172-175)
        FIIM_CUDA(launch_spmv(H, s, in, EpiScale{tm, IDv}, st, partials, fault));
        if (norm) FIIM_CUDA(launch_spmv(G, s, tm, EpiNorm{out}, st, partials, fault));
        else FIIM_CUDA(launch_spmv(G, s, tm, EpiStore{out}, st, partials, fault));
        return FIIM_OK;
    }
    // ACIFIM apply() mode 'C' (ACIFIM/src/bicgstab.cpp:395-404,408,411-420).
    FIIM_CUDA(launch_spmv(H, s, in, EpiStore{t1}, st, partials, fault));
    for (int it = 1; it < opt.nr; ++it) {
        FIIM_CUDA(launch_spmv(L, s, t1, EpiSubFrom{t3, in}, st, partials, fault));
        if (it == opt.nr - 1)
            FIIM_CUDA(launch_spmv(H, s, t3, EpiAccumScale{t1, t2, IDv}, st, partials, fault));
        else
            FIIM_CUDA(launch_spmv(H, s, t3, EpiAccum{t1}, st, partials, fault));
    }
    FIIM_CUDA(launch_spmv(G, s, t2, EpiStore{out}, st, partials, fault));
    for (int it = 1; it < opt.nr; ++it) {
        FIIM_CUDA(launch_spmv(U, s, out, EpiSubFrom{t3, t2}, st, partials, fault));
        if (it == opt.nr - 1 && norm)
            FIIM_CUDA(launch_spmv(G, s, t3, EpiAccumNorm{out}, st, partials, fault));
        else
            FIIM_CUDA(launch_spmv(G, s, t3, EpiAccum{out}, st, partials, fault));
    }
    return FIIM_OK;
}

int Solver::kernels_per_iteration() const {
    const bool combined = (opt.variant == FIIM_ACIFIM && opt.mode == 'C' && opt.nr > 1);
    const int prec = combined ? 2 + 4 * (opt.nr - 1) : 2;
    return 2 * prec + 5;
}

// One BiCGSTAB iteration (AFIIM/src/bicgstab.cpp:170-274) as launches on `stream`.
int Solver::enqueue_iteration(bool cond, cudaGraphConditionalHandle h) {
    cudaStream_t s = stream;
    const long nn = n;
    FIIM_TRY(enqueue_prec(p, pc, true));                                             // K1-K2
    FIIM_CUDA(launch_spmv(A, s, pc, EpiAlpha{v, r0}, st, partials, fault));     // K3
    FIIM_CUDA(launch_k(k_update_s<FinS>, stream_grid(k_update_s<FinS>, nn), 0, s, nn, r, v, x, sv, st, partials,
                       FinS{}));                                                        // K4
    FIIM_TRY(enqueue_prec(sv, sc, false));                                           // K5-K6
    FIIM_CUDA(launch_spmv(A, s, sc, EpiOmega{t, sv}, st, partials, fault));    // K7
    FIIM_CUDA(launch_k(k_update_xr<FinControl>, stream_grid(k_update_xr<FinControl>, nn), 0, s, nn, pc, sc, sv,
                       t, r0, x, r, st, partials, FinControl{}));                       // K8
    FIIM_CUDA(launch_k(k_update_p, stream_grid(k_update_p, nn), 0, s, nn, r, v, p, st, h, cond ? 1 : 0));  // K9
    return FIIM_OK;
}

int Solver::build_graph() {
    if (exec) {
        cudaGraphExecDestroy(exec);
        exec = nullptr;
    }
    if (graph) {
        cudaGraphDestroy(graph);
        graph = nullptr;
    }
    use_cond = false;
    // Run the body once with the state marked done (every kernel returns at once) so
    // launch shapes are resolved before capture begins.
    {
        DState h = {};
        h.done = 1;
        *hst = h;
        FIIM_CUDA(cudaMemcpyAsync(st, hst, sizeof(DState), cudaMemcpyHostToDevice, stream));
        FIIM_TRY(enqueue_iteration(false, cudaGraphConditionalHandle{}));
        FIIM_CUDA(cudaStreamSynchronize(stream));
    }
    // Preferred: one graph whose WHILE node repeats the iteration body on the device.
    // FIIM_GRAPH=host selects the host-driven graph (same kernels, same shapes), e.g.
    // for profilers that replay graph kernel nodes one by one.
    const char *mode_env = std::getenv("FIIM_GRAPH");
    const bool want_cond = !(mode_env && std::strcmp(mode_env, "host") == 0);
    do {
        if (!want_cond) break;
        cudaGraph_t g = nullptr;
        if (cudaGraphCreate(&g, 0) != cudaSuccess) break;
        cudaGraphConditionalHandle h;
        if (cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault) != cudaSuccess) {
            cudaGraphDestroy(g);
            break;
        }
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        if (cudaGraphAddNode(&node, g, nullptr, 0, &cp) != cudaSuccess) {
            cudaGraphDestroy(g);
            break;
        }
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        if (cudaStreamBeginCaptureToGraph(stream, body, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaGraphDestroy(g);
            break;
        }
        const int rc = enqueue_iteration(true, h);
        cudaGraph_t captured = nullptr;
        const cudaError_t ec = cudaStreamEndCapture(stream, &captured);
        if (rc != FIIM_OK || ec != cudaSuccess) {
            cudaGraphDestroy(g);
            break;
        }
        cudaGraphExec_t e = nullptr;
        if (cudaGraphInstantiate(&e, g, 0) != cudaSuccess) {
            cudaGraphDestroy(g);
            break;
        }
        graph = g;
        exec = e;
        use_cond = true;
    } while (0);
    cudaGetLastError();
    if (use_cond) return FIIM_OK;
    // Fallback: a graph of one iteration, relaunched by the host until done.
    FIIM_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    const int rc = enqueue_iteration(false, cudaGraphConditionalHandle{});
    cudaGraph_t g = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(stream, &g);
    if (rc != FIIM_OK) return rc;
    FIIM_CUDA(ec);
    FIIM_CUDA(cudaGraphInstantiate(&exec, g, 0));
    graph = g;
    return FIIM_OK;
}

// ------------------------------------------------------------------ set-up
int Solver::create(int n_, const int *Ai, const int *Aj, const double *Av, const int *Gi,
                   const int *Gj, const double *Gv, const double *IDv_, const int *Hi,
                   const int *Hj, const double *Hv, const int *Li, const int *Lj, const double *Lv,
                   const int *Ui, const int *Uj, const double *Uv, const fiim_options &o) {
    opt = o;
    n = n_;
    if (n <= 0 || !Ai || !Aj || !Av || !Gi || !Gj || !Gv || !IDv_)
        return set_error(FIIM_EARG, "null array or n <= 0");
    if (opt.variant < FIIM_AFIIM || opt.variant > FIIM_ACIFIM) return set_error(FIIM_EARG, "bad variant");
    if (opt.issym && opt.variant != FIIM_PDFIIM) return set_error(FIIM_EARG, "issym is a PDFIIM input form");
    if (opt.variant == FIIM_ACIFIM && opt.mode != 'E' && opt.mode != 'C')
        return set_error(FIIM_EARG, "ACIFIM mode '%c' is not the factored-inverse product (only 'E' and 'C')", opt.mode);
    const bool combined = (opt.variant == FIIM_ACIFIM && opt.mode == 'C' && opt.nr > 1);
    if (!opt.issym && (!Hi || !Hj || !Hv)) return set_error(FIIM_EARG, "H is required");
    if (combined && (!Li || !Lj || !Lv || !Ui || !Uj || !Uv)) return set_error(FIIM_EARG, "mode 'C' needs L and U");
    if (opt.precision != FIIM_FP64) return set_error(FIIM_EARG, "mixed precision is served by fiim_mixed_*");
    FIIM_TRY(check_device(&device));
    if (!stream) FIIM_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    const bool dev_src = (opt.memory == FIIM_MEM_DEVICE);

    // Host-side forms needed for symmetric input: full A and G^T.
    HostCsr Afull, Gt;
    std::vector<int> hA_rp, hA_ci, hG_rp, hG_ci;
    std::vector<double> hA_v, hG_v;
    const int *aRp = Ai, *aCi = Aj, *hRp = Hi, *hCi = Hj;
    const double *aV = Av, *hV = Hv;
    bool a_dev = dev_src, h_dev = dev_src;
    if (opt.issym) {
        auto fetch = [&](const int *rp, const int *ci, const double *v, std::vector<int> &orp,
                         std::vector<int> &oci, std::vector<double> &ov) -> int {
            orp.resize(n + 1);
            if (dev_src) FIIM_CUDA(cudaMemcpy(orp.data(), rp, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost));
            else std::memcpy(orp.data(), rp, sizeof(int) * (n + 1));
            const long z = orp[n];
            oci.resize(z);
            ov.resize(z);
            if (dev_src) {
                FIIM_CUDA(cudaMemcpy(oci.data(), ci, sizeof(int) * z, cudaMemcpyDeviceToHost));
                FIIM_CUDA(cudaMemcpy(ov.data(), v, sizeof(double) * z, cudaMemcpyDeviceToHost));
            } else {
                std::memcpy(oci.data(), ci, sizeof(int) * z);
                std::memcpy(ov.data(), v, sizeof(double) * z);
            }
            return FIIM_OK;
        };
        FIIM_TRY(fetch(Ai, Aj, Av, hA_rp, hA_ci, hA_v));
        FIIM_TRY(fetch(Gi, Gj, Gv, hG_rp, hG_ci, hG_v));
        expand_sym_upper(n, hA_rp.data(), hA_ci.data(), hA_v.data(), Afull);
        transpose_upper(n, hG_rp.data(), hG_ci.data(), hG_v.data(), Gt);
        aRp = Afull.rp.data(); aCi = Afull.ci.data(); aV = Afull.v.data(); a_dev = false;
        hRp = Gt.rp.data(); hCi = Gt.ci.data(); hV = Gt.v.data(); h_dev = false;
    }
    auto nnz_of = [&](const int *rp, bool dev) -> long {
        if (!dev) return rp[n];
        int z = 0;
        if (cudaMemcpy(&z, rp + n, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
        return z;
    };
    const long nA = nnz_of(aRp, a_dev), nG = nnz_of(Gi, dev_src), nH = nnz_of(hRp, h_dev);
    const long nL = combined ? nnz_of(Li, dev_src) : 0, nU = combined ? nnz_of(Ui, dev_src) : 0;
    if (nA < 0 || nG < 0 || nH < 0 || nL < 0 || nU < 0) return set_error(FIIM_ECUDA, "reading row offsets failed");

    const int nvec = combined ? 14 : 11;
    size_t bytes = csr_bytes(n, nA) + csr_bytes(n, nG) + csr_bytes(n, nH);
    if (combined) bytes += csr_bytes(n, nL) + csr_bytes(n, nU);
    bytes += (size_t)(nvec + 1) * Arena::need(sizeof(double) * n);
    const int max_blocks = num_sms() * 32;
    bytes += Arena::need(sizeof(DState)) + Arena::need(sizeof(double) * 4 * max_blocks) + Arena::need(16) + 1024;
    FIIM_TRY(arena.reserve(bytes));
    FIIM_TRY(carve_csr(arena, A, n, nA));
    FIIM_TRY(carve_csr(arena, G, n, nG));
    FIIM_TRY(carve_csr(arena, H, n, nH));
    if (combined) {
        FIIM_TRY(carve_csr(arena, L, n, nL));
        FIIM_TRY(carve_csr(arena, U, n, nU));
    }
    capA = nA; capG = nG; capH = nH; capL = nL; capU = nU;
    double **vecs[] = {&IDv, &x, &b, &r, &r0, &p, &v, &sv, &t, &pc, &sc, &tm, &t1, &t2, &t3};
    for (int k = 0; k < nvec + 1; ++k) {
        *vecs[k] = static_cast<double *>(arena.take(sizeof(double) * n));
        if (!*vecs[k]) return set_error(FIIM_ENOMEM, "arena exhausted");
    }
    st = static_cast<DState *>(arena.take(sizeof(DState)));
    partials = static_cast<double *>(arena.take(sizeof(double) * 4 * max_blocks));
    d_count = static_cast<unsigned long long *>(arena.take(sizeof(unsigned long long) * 5));
    fault = static_cast<int *>(arena.take(sizeof(int)));
    pbar = static_cast<unsigned *>(arena.take(16));
    if (!st || !partials || !d_count || !fault || !pbar) return set_error(FIIM_ENOMEM, "arena exhausted");
    if (!hst) FIIM_CUDA(cudaHostAlloc(&hst, sizeof(DState) + 128, cudaHostAllocDefault));
    h_count = reinterpret_cast<unsigned long long *>(reinterpret_cast<char *>(hst) + sizeof(DState) + 32);  // 5
    h_fault = reinterpret_cast<int *>(reinterpret_cast<char *>(hst) + sizeof(DState) + 80);
    FIIM_CUDA(cudaMemsetAsync(st, 0, sizeof(DState), stream));
    FIIM_CUDA(cudaMemsetAsync(fault, 0, sizeof(int), stream));

    if (dev_src) FIIM_CUDA(cudaMemcpyAsync(IDv, IDv_, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream));
    else FIIM_TRY(stager.copy(IDv, IDv_, sizeof(double) * n, stream));
    {
        DevCsr *mats[] = {&A, &G, &H, &L, &U};
        const long caps[] = {capA, capG, capH, capL, capU};
        const int *rps[] = {aRp, Gi, hRp, Li, Ui}, *cis[] = {aCi, Gj, hCi, Lj, Uj};
        const double *vs[] = {aV, Gv, hV, Lv, Uv};
        const int fills[] = {0, 1, 2, 2, 1};
        const bool dev[] = {a_dev, dev_src, h_dev, dev_src, dev_src};
        FIIM_TRY(upload_all(mats, caps, rps, cis, vs, fills, dev, combined ? 5 : 3, n, stream, d_count, h_count,
                             &stager));
    }

    DevCsr *mats[] = {&A, &G, &H, &L, &U};
    for (int k = 0; k < (combined ? 5 : 3); ++k) {
        DevCsr &M = *mats[k];
        if (opt.autotune) {
            FIIM_CUDA(cudaMemsetAsync(tm, 0, sizeof(double) * n, stream));
            FIIM_TRY(autotune_tile(M, tm, t, stream, fault));
        } else {
            // Deterministic shape: the same launch shape, hence the same reduction trees and
            // the same bits, in every process on the same GPU model. FIIM_SPMV=warp selects
            // the warp-block form instead.
            const char *form_env = std::getenv("FIIM_SPMV");
            if (form_env && std::strcmp(form_env, "warp") == 0) {
                M.form = kFormWarp;
                FIIM_TRY(set_tile(M, kWarpTile, stream));
            } else {
                M.form = kFormRows;
                FIIM_TRY(set_tile(M, default_tile(M), stream));
            }
        }
        FIIM_TRY(build_dia(M, stream));   // serves the products where the matrix allows it
    }
    {
        // FIIM_PERSIST=1: systems of at most kPersistMaxN rows solve as one cooperative launch.
        // Measured slower than the WHILE graph on B200 (Poisson 128^2: 41.7 against 34.7 us
        // per iteration), so it is not the default.
        const char *pe = std::getenv("FIIM_PERSIST");
        const bool want = pe && pe[0] == '1' && n <= kPersistMaxN;
        persistent = false;
        if (want && !combined) {
            int occ = 0, coop = 0;
            FIIM_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device));
            FIIM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_solve_persistent, kThreads, 0));
            const int most = std::max(A.nblk, std::max(G.nblk, H.nblk));
            const int max_blocks_p = num_sms() * 32;   // the partials buffer holds 2 x 4 per CTA
            persist_grid = std::min({occ * num_sms(), std::max(most, 1), max_blocks_p / 2});
            persistent = coop && occ > 0 && persist_grid > 0;
        }
        // Systems of at most kClusterCtas * kClusterMaxRows rows solve in one thread-block
        // cluster of kClusterCtas CTAs, where the device can run one (the default for them:
        // 21 against 35 us per iteration at n = 16,384); FIIM_PERSIST=0 keeps the WHILE graph,
        // FIIM_PERSIST=1 the cooperative launch.
        clustered = false;
        const bool cluster_ok = !pe || std::strcmp(pe, "cluster") == 0;
        if (cluster_ok && !persistent && !combined && n <= kClusterCtas * kClusterMaxRows) {
            cluster_rows = (n + kClusterCtas - 1) / kClusterCtas;
            const int smem = (int)cluster_smem(cluster_rows);
            FIIM_CUDA(cudaFuncSetAttribute(k_solve_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
            FIIM_CUDA(cudaFuncSetAttribute(k_solve_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
            cudaLaunchConfig_t cfg = {};
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = kClusterCtas;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.gridDim = dim3(kClusterCtas);
            cfg.blockDim = dim3(kClusterThreads);
            cfg.dynamicSmemBytes = smem;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            int clusters = 0;
            FIIM_CUDA(cudaOccupancyMaxActiveClusters(&clusters, k_solve_cluster, &cfg));
            clustered = clusters >= 1;
        }
    }
    FIIM_TRY(build_graph());
    if (!ev0) {
        FIIM_CUDA(cudaEventCreate(&ev0));
        FIIM_CUDA(cudaEventCreate(&ev1));
    }
    return FIIM_OK;
}

// Refill the values of an existing solver (same sizes); the graph stays valid because
// every buffer keeps its address.
int Solver::reload(const int *Ai, const int *Aj, const double *Av, const int *Gi, const int *Gj,
                   const double *Gv, const double *IDv_, const int *Hi, const int *Hj,
                   const double *Hv, const int *Li, const int *Lj, const double *Lv, const int *Ui,
                   const int *Uj, const double *Uv) {
    FIIM_CUDA(cudaSetDevice(device));
    const bool dev_src = (opt.memory == FIIM_MEM_DEVICE);
    const bool combined = (opt.variant == FIIM_ACIFIM && opt.mode == 'C' && opt.nr > 1);
    if (opt.issym) return set_error(FIIM_EARG, "reload does not serve symmetric input");
    if (dev_src) FIIM_CUDA(cudaMemcpyAsync(IDv, IDv_, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream));
    else FIIM_TRY(stager.copy(IDv, IDv_, sizeof(double) * n, stream));
    bool early[5] = {};   // refreshed on `aux` while the copies ran
    if (!aux && dia_wanted()) {
        FIIM_CUDA(cudaStreamCreateWithFlags(&aux, cudaStreamNonBlocking));
        for (cudaEvent_t &e : aux_ev) FIIM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        FIIM_CUDA(cudaHostAlloc(&h_spec, sizeof(int) * 5, cudaHostAllocDefault));
    }
    {
        DevCsr *mats[] = {&A, &G, &H, &L, &U};
        const long caps[] = {capA, capG, capH, capL, capU};
        const int *rps[] = {Ai, Gi, Hi, Li, Ui}, *cis[] = {Aj, Gj, Hj, Lj, Uj};
        const double *vs[] = {Av, Gv, Hv, Lv, Uv};
        const int fills[] = {0, 1, 2, 2, 1};
        const bool dev[] = {dev_src, dev_src, dev_src, dev_src, dev_src};
        auto issued = [&](int k) -> int {
            DevCsr &M = *mats[k];
            if (!aux || !M.rows_same || M.nblk <= 0 || !M.dia || M.dvbytes != 8) return FIIM_OK;
            early[k] = true;
            h_spec[k] = 1;
            return refresh_dia_async(M, stream, aux, aux_ev[k], h_spec + k);
        };
        const int rc = upload_all(mats, caps, rps, cis, vs, fills, dev, combined ? 5 : 3, n, stream, d_count,
                                  h_count, &stager, issued);
        if (aux) FIIM_CUDA(cudaStreamSynchronize(aux));
        if (rc != FIIM_OK) return rc;
    }
    // Row blocks follow the new row offsets (rebuilt only where they changed); the narrow
    // column stream follows the new column indices (rebuilt for every matrix: the same row
    // offsets may hold other columns). The graph bakes in each block count and stream width.
    bool regraph = false;
    DevCsr *mats[] = {&A, &G, &H, &L, &U};
    for (int k = 0; k < (combined ? 5 : 3); ++k) {
        DevCsr &M = *mats[k];
        const int old = M.nblk, was_narrow = M.narrow;
        // Everything of the sliced-diagonal copy that a captured launch holds: a rebuilt copy
        // may reuse the freed allocation's address with another layout inside it.
        auto dia_args = [](const DevCsr &D) {
            return std::make_tuple(D.dia, D.drec, D.dvals, D.nsl, D.drs, D.dsh);
        };
        const auto was_dia = dia_args(M);
        if (M.rows_same && M.nblk > 0) {
            // Refreshed early with the same columns: the narrow column stream still holds them.
            if (!(early[k] && h_spec[k] == 0)) {
                FIIM_TRY(build_narrow(M, stream));
                FIIM_TRY(refresh_dia(M, stream));
            }
        } else {
            FIIM_TRY(set_tile(M, M.tile, stream));
            FIIM_TRY(build_dia(M, stream));
        }
        regraph |= (M.nblk != old) || (M.narrow != was_narrow) || (dia_args(M) != was_dia);
    }
    if (regraph) FIIM_TRY(build_graph());
    return FIIM_OK;
}

// ------------------------------------------------------------------ solve
// solve_start enqueues the whole solve (input copies, start kernel, iteration graph, true
// residual) and returns while it runs (with the device-driven loop; the host-driven loop
// waits for it). solve_finish copies the scalars and x back and waits.
int Solver::solve_start(const double *b_in, const double *x_in, double tol, int nmax) {
    FIIM_CUDA(cudaSetDevice(device));
    const bool dev_src = (opt.memory == FIIM_MEM_DEVICE);
    const cudaMemcpyKind in_kind = dev_src ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    FIIM_CUDA(cudaEventRecord(ev0, stream));
    FIIM_CUDA(cudaMemsetAsync(fault, 0, sizeof(int), stream));
    if (inputs_staged) {
        inputs_staged = false;   // b and x0 went ahead of the matrices (stage_inputs)
    } else if (dev_src) {
        FIIM_CUDA(cudaMemcpyAsync(b, b_in, sizeof(double) * n, in_kind, stream));
        FIIM_CUDA(cudaMemcpyAsync(x, x_in, sizeof(double) * n, in_kind, stream));
    } else {
        FIIM_TRY(stager.copy(b, b_in, sizeof(double) * n, stream));
        FIIM_TRY(stager.copy(x, x_in, sizeof(double) * n, stream));
    }

    DState h = {};
    h.tol = tol;
    h.eps = 1.11022302462516e-16;                                    // AFIIM/src/bicgstab.cpp:108
    h.nmax = nmax;
    h.info = -1;
    if (opt.variant == FIIM_ACIFIM) h.maxmsteps = std::min(std::max(n, 2000) / 50, 40);  // ACIFIM :132
    else h.maxmsteps = std::min(std::max(n, 500) / 50, 20);                               // AFIIM :114
    h.alpha_guard = (opt.variant == FIIM_ACIFIM);
    *hst = h;
    FIIM_CUDA(cudaMemcpyAsync(st, hst, sizeof(DState), cudaMemcpyHostToDevice, stream));
    host_loops = 0;
    if (persistent) {
        pending_launches = 1;
        return launch_persistent();
    }
    if (clustered) {
        pending_launches = 1;
        return launch_cluster();
    }
    // Start: r = b - A x, r0 = r, p = r, ro = ||r0|| (AFIIM/src/bicgstab.cpp:151-165).
    FIIM_CUDA(launch_spmv(A, stream, x, EpiInit{b, p, r0, r}, st, partials, fault));
    pending_launches = 1;
    if (use_cond) {
        FIIM_CUDA(cudaGraphLaunch(exec, stream));
    } else {
        // Host-driven fallback: launch ahead in growing chunks; kernels of iterations
        // past termination return at once.
        int launched = 0, chunk = 1;
        for (;;) {
            for (int k = 0; k < chunk; ++k) FIIM_CUDA(cudaGraphLaunch(exec, stream));
            launched += chunk;
            FIIM_CUDA(cudaMemcpyAsync(&hst->done, &st->done, sizeof(int), cudaMemcpyDeviceToHost, stream));
            FIIM_CUDA(cudaStreamSynchronize(stream));
            if (hst->done) break;
            if (launched > std::max(nmax, 0) + 2)
                return set_error(FIIM_ETIMEOUT, "solve not finished after %d iterations", launched);
            chunk = std::min(chunk * 2, 16);
        }
        host_loops = launched;
    }
    // FP64 true residual ||b - A x|| / ||b||.
    FIIM_CUDA(launch_spmv(A, stream, x, EpiResid{b, nullptr}, st, partials, fault));
    pending_launches += 1;
    return FIIM_OK;
}

static PView pview(const DevCsr &M) {
    return PView{M.rp, M.ci, M.v, M.rb, M.eb, M.nblk, M.cd, M.cb, M.narrow};
}

int Solver::launch_persistent() {
    FIIM_CUDA(cudaMemsetAsync(pbar, 0, 16, stream));
    if (stall_next) {
        // Test hook: an arrival count that never reaches the grid size, so every CTA's first
        // barrier wait runs out and the solve returns FIIM_ETIMEOUT.
        const unsigned stuck[2] = {0x80000000u, 0u};
        FIIM_CUDA(cudaMemcpyAsync(pbar, stuck, sizeof(stuck), cudaMemcpyHostToDevice, stream));
        FIIM_CUDA(cudaStreamSynchronize(stream));
        stall_next = false;
    }
    PersistArgs a{pview(A), pview(G), pview(H), n, x, b, r, r0, p, v, sv, t, pc, sc, tm, IDv, st, partials, pbar,
                  fault, wait_limit};
    void *args[] = {&a};
    FIIM_CUDA(cudaLaunchCooperativeKernel((const void *)k_solve_persistent, dim3(persist_grid), dim3(kThreads), args, 0,
                                          stream));
    return FIIM_OK;
}

int Solver::launch_cluster() {
    ClusterArgs a{view(A), view(G), view(H), n, cluster_rows, x, b, IDv, st};
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kClusterCtas;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(kClusterCtas);
    cfg.blockDim = dim3(kClusterThreads);
    cfg.dynamicSmemBytes = cluster_smem(cluster_rows);
    cfg.stream = stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    FIIM_CUDA(cudaLaunchKernelEx(&cfg, k_solve_cluster, a));
    return FIIM_OK;
}

int Solver::solve_finish(double *x_io, fiim_result *res) {
    const bool dev_src = (opt.memory == FIIM_MEM_DEVICE);
    const cudaMemcpyKind out_kind = dev_src ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    FIIM_CUDA(cudaMemcpyAsync(hst, st, sizeof(DState), cudaMemcpyDeviceToHost, stream));
    FIIM_CUDA(cudaMemcpyAsync(h_fault, fault, sizeof(int), cudaMemcpyDeviceToHost, stream));
    if (x_io) FIIM_CUDA(cudaMemcpyAsync(x_io, x, sizeof(double) * n, out_kind, stream));
    FIIM_CUDA(cudaEventRecord(ev1, stream));
    FIIM_CUDA(cudaStreamSynchronize(stream));
    if (!use_cond) hst->loops = host_loops;
    float ms = 0.f;
    FIIM_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
    if (hst->info == -5) return set_error(FIIM_ETIMEOUT, "device loop guard tripped");
    if (*h_fault)
        return set_error(FIIM_ETIMEOUT, persistent ? "the solve's grid barrier did not complete within its limit"
                                                   : "a staged SpMV's bulk copy did not complete in time");
    const int launches = pending_launches + hst->loops * kernels_per_iteration();
    last_launches = launches;
    if (res) {
        res->resval = hst->rc / hst->ro;
        res->true_relres = std::sqrt(hst->ts) / std::sqrt(hst->tt);
        res->iter = hst->iter;
        res->info = hst->info;
        res->refine_steps = 0;
        res->device_ms = ms;
        res->launches = launches;
    }
    if (opt.verbose && x_io) print_status(hst->info, hst->iter, hst->rc / hst->ro);
    return FIIM_OK;
}

// Enqueues the copies of b and x0 that the next solve_start would make. The reference-facing
// call issues them before reload's matrix copies: a copy issued right after those copies and
// the refresh ran at under half the link's rate on B200 hosts (33.6 MB in 1.3-3.7 ms against
// 0.63 ms).
int Solver::stage_inputs(const double *b_in, const double *x_in) {
    FIIM_CUDA(cudaSetDevice(device));
    if (opt.memory == FIIM_MEM_DEVICE) {
        FIIM_CUDA(cudaMemcpyAsync(b, b_in, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream));
        FIIM_CUDA(cudaMemcpyAsync(x, x_in, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream));
    } else {
        FIIM_TRY(stager.copy(b, b_in, sizeof(double) * n, stream));
        FIIM_TRY(stager.copy(x, x_in, sizeof(double) * n, stream));
    }
    inputs_staged = true;
    return FIIM_OK;
}

int Solver::solve(const double *b_in, double *x_io, double tol, int nmax, fiim_result *res) {
    FIIM_TRY(solve_start(b_in, x_io, tol, nmax));
    return solve_finish(x_io, res);
}

// The reference's termination messages (AFIIM/src/bicgstab.cpp:227-252,279-280;
// PDFIIM prints its divergence text on stagnation too, PDFIIM/src/bicgstab.cpp:257-261).
void Solver::print_status(int info, int iter, double rel) const {
    if (info == 1 || (info == 2 && opt.variant == FIIM_PDFIIM)) {
        std::cout << "BiCGSTAB diverged and iterations stopped with relative residual " << rel
                  << " in iteration " << iter << "\n";
        std::cout << "Try to increase the quality of preconditioning\n";
    } else if (info == 2) {
        std::cout << "BiCGSTAB stagnated with relative residual " << rel << " in iteration " << iter << "\n";
        std::cout << "Try increasing prescribed tolerance\n";
    } else if (info == 0) {
        std::cout << "Convergence in " << iter << " iterations with relative residual " << rel << "\n";
    }
    if (info == 3)
        std::cout << "Convergence failed after " << iter << " iterations with relative residual " << rel << "\n";
}

void Solver::destroy() {
    if (device >= 0) cudaSetDevice(device);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    ev0 = ev1 = nullptr;
    if (stream) cudaStreamDestroy(stream);
    stream = nullptr;
    if (aux) cudaStreamDestroy(aux);
    aux = nullptr;
    for (cudaEvent_t &e : aux_ev) {
        if (e) cudaEventDestroy(e);
        e = nullptr;
    }
    if (h_spec) cudaFreeHost(h_spec);
    h_spec = nullptr;
    if (hst) cudaFreeHost(hst);
    hst = nullptr;
    stager.release();
    for (DevCsr *M : {&A, &G, &H, &L, &U}) release_dia(*M);
    arena.release();
}

// ------------------------------------------------------------------ single products
// y = A x (op 0) or y = M x with the solver's preconditioner (op 1), using the
// solver's own tuned kernels. x and y live in opt.memory space.
int Solver::apply(int op, const double *in, double *out) {
    FIIM_CUDA(cudaSetDevice(device));
    if (op != 0 && op != 1) return set_error(FIIM_EARG, "op is 0 (A) or 1 (preconditioner)");
    const bool dev_src = (opt.memory == FIIM_MEM_DEVICE);
    FIIM_CUDA(cudaMemcpyAsync(sv, in, sizeof(double) * n,
                              dev_src ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, stream));
    DState h = {};
    *hst = h;
    FIIM_CUDA(cudaMemcpyAsync(st, hst, sizeof(DState), cudaMemcpyHostToDevice, stream));
    if (op == 0) FIIM_CUDA(launch_spmv(A, stream, sv, EpiStore{t}, st, partials, fault));
    else FIIM_TRY(enqueue_prec(sv, t, false));
    FIIM_CUDA(cudaMemcpyAsync(out, t, sizeof(double) * n,
                              dev_src ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, stream));
    FIIM_CUDA(cudaStreamSynchronize(stream));
    return FIIM_OK;
}

// ------------------------------------------------------------------ per-kernel timing
// Replays each launch of the iteration body on its own, `reps` times, between CUDA
// events on the solver's stream, after a solve has left the vectors populated. The
// scalars are reset so no kernel takes its early exit. Reports the mean device ms of
// each launch and its algorithmic bytes: a matrix pass S(M) = nnz*(8+4) + 4*(n+1),
// one read of the gathered vector, and every other vector read or written once.
int Solver::kernel_times(int reps, int max_k, double *ms, double *bytes, char *names, int name_len,
                         bool in_sequence, double *body_ms) {
    FIIM_CUDA(cudaSetDevice(device));
    const bool combined = (opt.variant == FIIM_ACIFIM && opt.mode == 'C' && opt.nr > 1);
    if (combined) return set_error(FIIM_EARG, "kernel timing covers mode 'E' bodies");
    struct Item { const char *name; double bytes; std::function<cudaError_t()> go; };
    const double nv = 8.0 * n;
    auto S = [&](const DevCsr &M) { return 12.0 * M.nnz + 4.0 * (M.n + 1); };
    const long nn = n;
    std::vector<Item> items = {
        {"H_spmv_scale", S(H) + 3 * nv, [&] { return launch_spmv(H, stream, p, EpiScale{tm, IDv}, st, partials, fault); }},
        {"G_spmv_norm", S(G) + 2 * nv, [&] { return launch_spmv(G, stream, tm, EpiNorm{pc}, st, partials, fault); }},
        {"A_spmv_alpha", S(A) + 3 * nv, [&] { return launch_spmv(A, stream, pc, EpiAlpha{v, r0}, st, partials, fault); }},
        {"update_s", 4 * nv, [&] { k_update_s<FinS><<<stream_grid(k_update_s<FinS>, nn), kThreads, 0, stream>>>(nn, r, v, x, sv, st, partials, FinS{}); return cudaGetLastError(); }},
        {"G_spmv", S(G) + 2 * nv, [&] { return launch_spmv(G, stream, tm, EpiStore{sc}, st, partials, fault); }},
        {"A_spmv_omega", S(A) + 3 * nv, [&] { return launch_spmv(A, stream, sc, EpiOmega{t, sv}, st, partials, fault); }},
        {"update_xr", 8 * nv, [&] { k_update_xr<FinControl><<<stream_grid(k_update_xr<FinControl>, nn), kThreads, 0, stream>>>(nn, pc, sc, sv, t, r0, x, r, st, partials, FinControl{}); return cudaGetLastError(); }},
        {"update_p", 4 * nv, [&] { k_update_p<<<stream_grid(k_update_p, nn), kThreads, 0, stream>>>(nn, r, v, p, st, cudaGraphConditionalHandle{}, 0); return cudaGetLastError(); }},
    };
    if (in_sequence)   // the body's second H product (K5), between the s update and G's product
        items.insert(items.begin() + 4, Item{"H_spmv_scale", S(H) + 3 * nv, [&] {
            return launch_spmv(H, stream, sv, EpiScale{tm, IDv}, st, partials, fault); }});
    // Scalars that keep every kernel on its full path; the solver's vectors are
    // scratch here (each solve starts from the caller's x and b).
    DState h = {};
    h.tol = 0.0; h.eps = 0.0; h.nmax = 1 << 30; h.maxmsteps = 1 << 30; h.info = -1;
    h.m1 = 1.0; h.alpha = 1e-30; h.omega = 1e-30; h.beta = 1e-30; h.ro = 1.0; h.rc = 1.0;
    *hst = h;
    FIIM_CUDA(cudaMemcpyAsync(st, hst, sizeof(DState), cudaMemcpyHostToDevice, stream));
    const int k = std::min<int>((int)items.size(), max_k);
    if (in_sequence) {
        // The body in order, an event between consecutive launches; then the same body
        // without the events in between, for the events' own cost.
        std::vector<cudaEvent_t> ev(k + 1);
        for (auto &e : ev) FIIM_CUDA(cudaEventCreate(&e));
        std::vector<double> acc(k, 0.0);
        for (int i = 0; i < k; ++i) FIIM_CUDA(items[i].go());   // warm
        for (int rr = 0; rr < reps; ++rr) {
            for (int i = 0; i < k; ++i) {
                FIIM_CUDA(cudaEventRecord(ev[i], stream));
                FIIM_CUDA(items[i].go());
            }
            FIIM_CUDA(cudaEventRecord(ev[k], stream));
            FIIM_CUDA(cudaEventSynchronize(ev[k]));
            for (int i = 0; i < k; ++i) {
                float t_ms = 0.f;
                FIIM_CUDA(cudaEventElapsedTime(&t_ms, ev[i], ev[i + 1]));
                acc[i] += t_ms;
            }
        }
        FIIM_CUDA(cudaEventRecord(ev[0], stream));
        for (int rr = 0; rr < reps; ++rr)
            for (int i = 0; i < k; ++i) FIIM_CUDA(items[i].go());
        FIIM_CUDA(cudaEventRecord(ev[k], stream));
        FIIM_CUDA(cudaEventSynchronize(ev[k]));
        float whole = 0.f;
        FIIM_CUDA(cudaEventElapsedTime(&whole, ev[0], ev[k]));
        if (body_ms) *body_ms = whole / reps;
        for (auto &e : ev) cudaEventDestroy(e);
        for (int i = 0; i < k; ++i) {
            ms[i] = acc[i] / reps;
            bytes[i] = items[i].bytes;
            if (names) std::snprintf(names + (size_t)i * name_len, name_len, "%s", items[i].name);
        }
        return k;
    }
    for (int i = 0; i < k; ++i) {
        FIIM_CUDA(items[i].go());   // warm
        FIIM_CUDA(cudaEventRecord(ev0, stream));
        for (int rr = 0; rr < reps; ++rr) FIIM_CUDA(items[i].go());
        FIIM_CUDA(cudaEventRecord(ev1, stream));
        FIIM_CUDA(cudaEventSynchronize(ev1));
        float t_ms = 0.f;
        FIIM_CUDA(cudaEventElapsedTime(&t_ms, ev0, ev1));
        ms[i] = t_ms / reps;
        bytes[i] = items[i].bytes;
        if (names) std::snprintf(names + (size_t)i * name_len, name_len, "%s", items[i].name);
    }
    return k;
}

double Solver::iteration_bytes() const {
    // One iteration of the reference's algorithm: every matrix streamed twice, 32 vector
    // passes (the compulsory reads and writes of AFIIM/src/bicgstab.cpp:170-271).
    auto S = [&](const DevCsr &M) { return 12.0 * M.nnz + 4.0 * (M.n + 1); };
    return 2 * S(A) + 2 * S(G) + 2 * S(H) + 32.0 * 8.0 * n;
}

// ------------------------------------------------------------------ kernel-level API
int spmv_api(int n, const int *Ai, const int *Aj, const double *Av, const double *x, double *y,
             int vec, cudaStream_t s) {
    if (n <= 0 || !Ai || !Aj || !Av || !x || !y) return set_error(FIIM_EARG, "null array or n <= 0");
    FIIM_TRY(check_device(nullptr));
    if (vec != 2 && vec != 4 && vec != 8 && vec != 16 && vec != 32) {
        int z = 0;
        FIIM_CUDA(cudaMemcpyAsync(&z, Ai + n, sizeof(int), cudaMemcpyDeviceToHost, s));
        FIIM_CUDA(cudaStreamSynchronize(s));
        vec = heuristic_vec(n, z);
    }
    FIIM_CUDA(launch_spmv_vec(vec, s, CsrView<double>{Ai, Aj, Av, n}, x, EpiStore{y}, nullptr, nullptr));
    return FIIM_OK;
}

int prec_api(int n, const int *Gi, const int *Gj, const double *Gv, const double *IDv_, const int *Hi,
             const int *Hj, const double *Hv, const double *rr, double *z, double *tmv, cudaStream_t s) {
    if (n <= 0 || !Gi || !Gj || !Gv || !IDv_ || !Hi || !Hj || !Hv || !rr || !z || !tmv)
        return set_error(FIIM_EARG, "null array or n <= 0");
    FIIM_TRY(check_device(nullptr));
    int zz[2] = {0, 0};
    FIIM_CUDA(cudaMemcpyAsync(&zz[0], Gi + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    FIIM_CUDA(cudaMemcpyAsync(&zz[1], Hi + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    FIIM_CUDA(cudaStreamSynchronize(s));
    FIIM_CUDA(launch_spmv_vec<2>(heuristic_vec(n, zz[1]), s, CsrView<double>{Hi, Hj, Hv, n}, rr,
                             EpiScale{tmv, IDv_}, nullptr, nullptr));
    FIIM_CUDA(launch_spmv_vec<1>(heuristic_vec(n, zz[0]), s, CsrView<double>{Gi, Gj, Gv, n}, tmv,
                             EpiStore{z}, nullptr, nullptr));
    return FIIM_OK;
}

}  // namespace fiim
