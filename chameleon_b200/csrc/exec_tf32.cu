// exec_tf32.cu -- executor kernel variant: FP32 tiles, TF32x3 products on mma.sync.
#include "executor_kernel.cuh"

namespace chb {
int launch_dag_tf32(const ExecParams &p, int grid, cudaStream_t s) { return launch_dag<float, SPLIT_TF32X3, false>(p, grid, s); }
}  // namespace chb
