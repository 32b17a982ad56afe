// Mixed-precision solve: FP64 iterative refinement around an FP32 inner BiCGSTAB.
#include "fiim_b200.h"
#include "fiim_internal.h"
#include "fiim_solver.h"

int fiim_is_mixed(fiim_solver_t h) {
    return h && reinterpret_cast<fiim::SolverBase *>(h)->kind == fiim::kKindMixed;
}
int fiim_mixed_create(fiim_solver_t *, int, const int *, const int *, const double *, const int *,
                      const int *, const double *, const double *, const int *, const int *,
                      const double *, const fiim_options *) {
    return fiim::set_error(FIIM_EARG, "mixed precision not available in this build");
}
int fiim_mixed_solve(fiim_solver_t, const double *, double *, double, int, fiim_result *) {
    return fiim::set_error(FIIM_EARG, "mixed precision not available in this build");
}
int64_t fiim_mixed_device_bytes(fiim_solver_t) { return -1; }
int fiim_mixed_destroy(fiim_solver_t) { return FIIM_OK; }
