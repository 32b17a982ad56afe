// Internal declarations shared by the host-side translation units.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include <cstdarg>
#include <cstdlib>
#include <algorithm>
#include <cstddef>
#include <map>
#include <mutex>
#include <vector>

#include "fiim_b200.h"

namespace fiim {

int set_error(int code, const char *fmt, ...);
const char *last_error();
int check_device(int *dev_out);
int num_sms();

#define FIIM_CUDA(call)                                                                   \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            cudaGetLastError();                                                           \
            return ::fiim::set_error(FIIM_ECUDA, "%s: %s (%s:%d)", #call,                 \
                                     cudaGetErrorString(e_), __FILE__, __LINE__);         \
        }                                                                                 \
    } while (0)

#define FIIM_TRY(call)                      \
    do {                                    \
        int rc_ = (call);                   \
        if (rc_ != FIIM_OK) return rc_;     \
    } while (0)

// One device allocation carved into 256-byte aligned pieces.
struct Arena {
    void *base = nullptr;
    size_t cap = 0, used = 0;
    int reserve(size_t bytes);   // ensure capacity (reallocates only to grow); resets use
    void *take(size_t bytes);    // nullptr when exhausted
    void release();
    static size_t need(size_t bytes);
};

// Forms of the solver's SpMV. All give the same bits. The CSR-stream forms differ in how a
// row block's streams reach shared memory: through registers, pipelined by one block
// (kFormRows, fiim_kernels.cuh), by bulk copies into two buffers (kFormBulk, fiim_pipe.cuh),
// or per warp (kFormWarp); kFormDia reads the sliced-diagonal copy of the values instead.
constexpr int kFormRows = 0, kFormBulk = 1, kFormWarp = 2, kFormDia = 3;

// A CSR matrix resident on the device. v holds FP64 values; v32 / v16 are optional
// FP32 / BF16 copies for the mixed-precision inner solve.
struct DevCsr {
    long n = 0, nnz = 0;
    int *rp = nullptr, *ci = nullptr;
    double *v = nullptr;
    float *v32 = nullptr;
    __nv_bfloat16 *v16 = nullptr;
    int vec = 8;                 // lanes per row of the set-up-free SpMV
    int tile = 2048;             // entries per row block of the CSR-stream SpMV
    int form = 0;                // CSR-stream SpMV form, one of the kForm* constants
    int *rb = nullptr;           // row-block first rows (device), nblk + 1 entries
    int *eb = nullptr;           // row-block first entries (device), nblk + 1 entries
    int *cb = nullptr;           // row-block base columns of the narrow column stream
    short *cd = nullptr;         // narrow column stream: column - block base (device)
    int *wide = nullptr;         // device flag written by the narrow-stream builder
    int narrow = 0;              // 1: the CSR-stream SpMV reads cd / cb instead of ci
    int nblk = 0;
    // Sliced-diagonal copy (kFormDia; fiim_kernels.cuh, k_spmv_dia), in its own allocation.
    int dia = 0;                 // 1: built and current
    int nsl = 0;                 // slices of dsh rows
    int dsh = 0;                 // rows a slice: 32 R, R rows a lane (dia_rows_per_lane)
    int drs = 0;                 // ints per slice record (16 or 32): first diagonal, count, offsets
    long ndiag = 0;              // diagonals over all slices (dsh slots each)
    int *drec = nullptr;         // nsl records
    int *dmap = nullptr;         // nnz: the slot of each entry
    int *dbad = nullptr;         // device flag of the structure check and value placement
    void *dvals = nullptr;       // dsh * ndiag values of dvbytes bytes each (FP64, FP32 or BF16)
    int dvbytes = 0;
    void *dia_mem = nullptr;
    size_t dia_bytes = 0;        // size of that allocation
    bool dia_tried = false;      // the copy was considered for the columns hashed in dia_cols
    unsigned long long dia_cols = 0;
    unsigned long long *dhash = nullptr;   // device scratch of the column hash (in the arena)
    std::vector<int> hseg_sl;    // first slice of each segment (host), segments + 1 entries
    bool dseg = false;           // built with several segments: only the batched kernel reads it
    std::vector<int> hrp;        // row offsets on the host (row blocks, tuning key)
    bool rows_same = false;      // the last upload_csr found the same row offsets as before
    std::vector<long> sig;       // tuning-cache key: n, nnz, sampled row offsets
};

// Row blocks of a CSR matrix: consecutive rows, at most max_rows of them, whose entries
// total at most tile; a row with more than tile entries forms a block by itself.
void build_row_blocks(const std::vector<int> &rp, int tile, int max_rows, std::vector<int> &rb);

// Host CSR (owning), used for symmetric expansion and transposes.
struct HostCsr {
    int n = 0;
    std::vector<int> rp, ci;
    std::vector<double> v;
};

int heuristic_vec(long n, long nnz);

// Set-up helpers shared by the FP64 and mixed-precision solvers (fiim_solver.cu).
void signature(DevCsr &M, const int *host_rp);
size_t csr_bytes(long n, long nnz);
int carve_csr(Arena &ar, DevCsr &M, long n, long nnz);
// Host-to-device copies from pageable memory through a ring of pinned buffers: a chunk is
// copied into a pinned buffer by all host threads while the previous chunks' DMA runs, which
// moves pageable data several times faster than a copy from pageable memory (staged by the
// driver one page run at a time). Pinned sources and small copies go straight to
// cudaMemcpyAsync. As with that call, the source is read completely before copy() returns;
// the DMA from the pinned buffers may still be in flight.
struct Stager {
    static constexpr int kBufs = 4;
    static constexpr size_t kChunk = size_t(16) << 20;
    static constexpr size_t kMinStaged = size_t(4) << 20;
    void *buf[kBufs] = {};
    cudaEvent_t ev[kBufs] = {};
    bool pending[kBufs] = {};
    int next = 0;
    int copy(void *dst, const void *src, size_t bytes, cudaStream_t s);
    void release();
};

int upload_csr_async(DevCsr &M, long nnz_cap, int n, const int *rp, const int *ci, const double *v, bool device_src,
                     cudaStream_t s, Stager *stager = nullptr);
int check_fill_launch(DevCsr &M, int fill, cudaStream_t s, unsigned long long *d_count, unsigned long long *h_count);
int check_fill_finish(DevCsr &M, int fill, unsigned long long outside);
int upload_csr(DevCsr &M, long nnz_cap, int n, const int *rp, const int *ci, const double *v, int fill,
               bool device_src, cudaStream_t s, unsigned long long *d_count, unsigned long long *h_count);
int set_tile(DevCsr &M, int tile, cudaStream_t s);
// Builds the narrow column stream (cd, cb) of M's row blocks (eb) when every block allows it.
int build_narrow(DevCsr &M, cudaStream_t s);
// The sliced-diagonal copy of M (fiim_kernels.cuh, k_spmv_dia). build_dia_structure lays it
// out (slice records, the slot of every entry; slices never straddle a boundary of
// `segments`, ascending row starts from 0 to n, one segment when null) for values of vbytes
// bytes (8, 4 or 2) when
// M's rows are sorted by column, every slice (32 R rows, R = dia_rows_per_lane) has at most
// kDiaMaxDiags diagonals and the copy moves fewer bytes than the CSR streams (M.dia_mem
// stays null otherwise);
// place_dia moves the nnz values `vals` (device, that width) into it and sets M.dia = 1,
// unless an entry holds the padding pattern (then the copy is released). dia_fits tells
// whether M's current columns (same row offsets) still sit in the laid-out slots.
// build_dia / refresh_dia do this for the FP64 values M.v: refresh_dia, after new values (and
// possibly new columns) with the same row offsets, re-places the values when the columns
// still fit and rebuilds otherwise. release_dia frees the copy; dia_wanted is false under
// FIIM_DIA=0 or FIIM_SPMV=rows / staged / warp.
bool dia_wanted();
// Rows a lane of the sliced-diagonal copy for values of vbytes bytes: 2 for FP32, 4 for BF16;
// for FP64 0, which lets build_dia_structure choose 1 or 2 by the matrix (FIIM_DIA_R=1 or 2
// forces one).
int dia_rows_per_lane(int vbytes);

int build_dia_structure(DevCsr &M, cudaStream_t s, int vbytes, const std::vector<int> *segments = nullptr);
int place_dia(DevCsr &M, const void *vals, cudaStream_t s);
int dia_fits(DevCsr &M, cudaStream_t s, bool *fits);
int build_dia(DevCsr &M, cudaStream_t s);
int refresh_dia(DevCsr &M, cudaStream_t s);
void release_dia(DevCsr &M);
void expand_sym_upper(int n, const int *rp, const int *ci, const double *v, HostCsr &out);
void transpose_upper(int n, const int *rp, const int *ci, const double *v, HostCsr &out);

// Launch a 256-thread kernel with programmatic stream serialization (programmatic
// dependent launch: the kernel's CTAs may be scheduled while the previous kernel in the
// stream finishes; the kernels wait for it with griddepcontrol.wait before touching its
// results). FIIM_PDL=0 launches without the attribute.
inline bool pdl_enabled() {
    static const bool on = [] {
        const char *e = std::getenv("FIIM_PDL");
        return !(e && e[0] == '0' && e[1] == 0);
    }();
    return on;
}

template <typename... KArgs, typename... Args>
cudaError_t launch_k(void (*kern)(KArgs...), int grid, size_t smem, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

// Resident blocks per SM of a kernel launched with 256 threads, cached by kernel address.
template <typename K>
int occupancy(K kernel) {
    constexpr int kBlockThreads = 256;
    static std::mutex mu;
    static std::map<const void *, int> occ;
    std::lock_guard<std::mutex> lk(mu);
    auto it = occ.find((const void *)kernel);
    if (it != occ.end()) return it->second;
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, kBlockThreads, 0) != cudaSuccess || b < 1) {
        cudaGetLastError();
        b = 4;
    }
    occ[(const void *)kernel] = b;
    return b;
}

// Grid: enough blocks for the work, capped at one full wave of resident blocks.
template <typename K>
int grid_for(K kernel, long units_per_block, long units) {
    const long need = std::max<long>(1, (units + units_per_block - 1) / units_per_block);
    return (int)std::min<long>(need, (long)occupancy(kernel) * num_sms());
}


}  // namespace fiim
