// exec_f32tc.cu -- executor kernel variant: FP32 tiles, BF16x3 trailing updates on tcgen05.
#include "executor_kernel.cuh"

namespace chb {
int launch_dag_f32tc(const ExecParams &p, int grid, cudaStream_t s) { return launch_dag<float, SPLIT_BF16X3, true>(p, grid, s); }
}  // namespace chb
