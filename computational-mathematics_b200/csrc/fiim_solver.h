// The FP64 solver object behind fiim_solver_t and the reference-facing drop-ins.
#pragma once

#include <cuda_runtime.h>

#include "fiim_b200.h"
#include "fiim_internal.h"
#include "fiim_kernels.cuh"

namespace fiim {

// Every handle starts with its kind so the C-ABI can dispatch on it.
enum { kKindFp64 = 0x46503634, kKindMixed = 0x4d495844 };
struct SolverBase {
    int kind;
};

struct Solver : SolverBase {
    Solver() { kind = kKindFp64; }
    int device = -1;
    int n = 0;
    fiim_options opt{};
    cudaStream_t stream = nullptr;
    Arena arena;
    DevCsr A, G, H, L, U;        // H is G^T for symmetric PDFIIM input
    long capA = 0, capG = 0, capH = 0, capL = 0, capU = 0;
    double *IDv = nullptr;
    double *x = nullptr, *b = nullptr, *r = nullptr, *r0 = nullptr, *p = nullptr, *v = nullptr;
    double *sv = nullptr, *t = nullptr, *pc = nullptr, *sc = nullptr, *tm = nullptr;
    double *t1 = nullptr, *t2 = nullptr, *t3 = nullptr;   // ACIFIM mode 'C' work vectors
    DState *st = nullptr;        // device scalars
    DState *hst = nullptr;       // pinned host mirror
    double *partials = nullptr;  // per-block reduction partials
    unsigned long long *d_count = nullptr, *h_count = nullptr;
    int *h_fault = nullptr;
    int *fault = nullptr;        // raised by a staged SpMV whose bulk copy did not complete
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool use_cond = false;       // the graph holds a device-driven WHILE loop
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int last_launches = 0;

    int create(int n, const int *Ai, const int *Aj, const double *Av, const int *Gi, const int *Gj,
               const double *Gv, const double *IDv, const int *Hi, const int *Hj, const double *Hv,
               const int *Li, const int *Lj, const double *Lv, const int *Ui, const int *Uj,
               const double *Uv, const fiim_options &o);
    int reload(const int *Ai, const int *Aj, const double *Av, const int *Gi, const int *Gj,
               const double *Gv, const double *IDv, const int *Hi, const int *Hj, const double *Hv,
               const int *Li, const int *Lj, const double *Lv, const int *Ui, const int *Uj,
               const double *Uv);
    int solve(const double *b, double *x, double tol, int nmax, fiim_result *res);
    // The two halves of solve: enqueue (returns while the device-driven loop runs), then copy
    // the scalars and x (x_io == NULL: discard the result) and wait.
    int solve_start(const double *b, const double *x, double tol, int nmax);
    int solve_finish(double *x_io, fiim_result *res);
    int pending_launches = 0, host_loops = 0;
    Stager stager;               // host-to-device copies from pageable memory
    // The reference-facing call's reload: b and x0 are copied ahead of the matrices
    // (stage_inputs; the next solve_start then copies no inputs), and each sliced-diagonal
    // copy is refreshed on the second stream `aux` while the later matrices' copies run.
    bool inputs_staged = false;
    int stage_inputs(const double *b, const double *x);
    cudaStream_t aux = nullptr;
    cudaEvent_t aux_ev[5] = {};
    int *h_spec = nullptr;       // pinned: per matrix, the flag of its refresh on `aux`
    // Small systems: the whole solve as one cooperative launch (fiim_persist.cuh).
    bool persistent = false;
    int persist_grid = 0;
    // Small systems: the whole solve in one thread-block cluster, vectors in shared memory
    // (fiim_cluster.cuh).
    bool clustered = false;
    int cluster_rows = 0;
    int launch_cluster();
    unsigned *pbar = nullptr;    // grid barrier words
    int wait_limit = 1 << 21;    // barrier polls (back-to-back acquire loads of the barrier word) before a solve gives up
    bool stall_next = false;     // test hook: the next solve's first barrier never completes
    int launch_persistent();
    void destroy();
    size_t device_bytes() const {   // the arena and the sliced-diagonal copies
        return arena.cap + A.dia_bytes + G.dia_bytes + H.dia_bytes + L.dia_bytes + U.dia_bytes;
    }

    int enqueue_prec(const double *in, double *out, bool norm);
    int enqueue_iteration(bool cond, cudaGraphConditionalHandle h);
    int build_graph();
    int kernels_per_iteration() const;
    void print_status(int info, int iter, double rel) const;
    int apply(int op, const double *in, double *out);
    int kernel_times(int reps, int max_k, double *ms, double *bytes, char *names, int name_len,
                     bool in_sequence = false, double *body_ms = nullptr);
    double iteration_bytes() const;
};

}  // namespace fiim

// Mixed-precision solver (fiim_mixed.cu).
int fiim_is_mixed(fiim_solver_t h);
int fiim_mixed_create(fiim_solver_t *out, int n, const int *Ai, const int *Aj, const double *Av,
                      const int *Gi, const int *Gj, const double *Gv, const double *IDv,
                      const int *Hi, const int *Hj, const double *Hv, const fiim_options *opt);
int fiim_mixed_solve(fiim_solver_t h, const double *b, double *x, double tol, int NMAX,
                     fiim_result *res);
int64_t fiim_mixed_device_bytes(fiim_solver_t h);
int fiim_mixed_destroy(fiim_solver_t h);

namespace fiim {

int spmv_api(int n, const int *Ai, const int *Aj, const double *Av, const double *x, double *y,
             int vec, cudaStream_t s);
int prec_api(int n, const int *Gi, const int *Gj, const double *Gv, const double *IDv,
             const int *Hi, const int *Hj, const double *Hv, const double *r, double *z,
             double *tm, cudaStream_t s);

}  // namespace fiim
