// exec_f32.cu -- executor kernel variant: FP32 tiles, BF16x3 products on mma.sync.
#include "executor_kernel.cuh"

namespace chb {
int launch_dag_f32(const ExecParams &p, int grid, cudaStream_t s) { return launch_dag<float, SPLIT_BF16X3, false>(p, grid, s); }
}  // namespace chb
