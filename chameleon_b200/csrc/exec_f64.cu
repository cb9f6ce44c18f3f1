// exec_f64.cu -- executor kernel variant: FP64 tiles (DMMA).
#include "executor_kernel.cuh"

namespace chb {
int launch_dag_f64(const ExecParams &p, int grid, cudaStream_t s) { return launch_dag<double, SPLIT_BF16X3, false>(p, grid, s); }
}  // namespace chb
