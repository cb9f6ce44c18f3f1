// noalloc.cu -- CUDA_dpotrf_noalloc: the diagonal-tile Cholesky without any
// device allocation.
//
// CUDA_dpotrf keeps its scratch (the inverted 64 x 64 diagonal blocks of the
// factor) in a buffer that the handle grows with cudaMalloc on demand.  Some
// callers cannot allow that: a task runtime that owns all device memory and
// forbids allocations inside its worker callbacks (a StarPU codelet, for
// instance), code that must not pay the implicit device synchronization and
// latency that cudaMalloc/cudaFree can bring, or an application that reserves
// its whole memory budget up front.  This entry point uses instead one
// fixed-size scratch array in the library's own device memory, so a call only
// launches a kernel.
//
// Limits and sharing:
//  * n <= CHAM_B200_NOALLOC_POTRF_MAXN (1024); larger n is rejected with
//    CHAMELEON_ERR_INTERNAL_LIMIT before anything is launched.
//  * The array (512 KiB) exists on every GPU that loads the library and stays
//    allocated until the process exits.
//  * All calls on a device share it: calls whose kernels can overlap on the GPU
//    (different streams, no ordering between them) race on it and must not be
//    issued.  Calls on one stream are ordered and safe.
//  * The first call on a device looks up the array's device address
//    (cudaGetSymbolAddress) with that device current and sets the kernel's
//    shared-memory limit; make that first call before any stream capture.
//  * The array keeps the last call's contents; nothing in it needs to start at
//    zero (every block is written before it is read).
#include <cuda_runtime.h>

#include <mutex>

#include "core.cuh"
#include "internal.h"
#include "rec.cuh"

#define CHAM_B200_NOALLOC_POTRF_MAXN 1024

namespace chb {

static __device__ __align__(256) double g_potrf_scratch[(CHAM_B200_NOALLOC_POTRF_MAXN / IB) * IB * IB];

// The same tile algorithm as CUDA_dpotrf's kernel (blocked left-looking with
// the 64-wide leaf), so both entry points return the same factor and info.
__global__ void __launch_bounds__(NT_CTA, 1) potrf_noalloc_kernel(View T, int n, double *invd, int *info) {
    extern __shared__ __align__(128) double smem[];
    const int r = rec::tile_potrf_blk<double, SPLIT_BF16X3>(T, n, invd, smem);
    if (threadIdx.x == 0 && info) *info = r;
}

namespace {
constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
double *g_scratch_addr[MAX_DEVICES] = {};
bool g_attr_set[MAX_DEVICES] = {};

// Per-device set-up: device address of the scratch array, kernel attribute.
int noalloc_setup(int dev, double **addr) {
    if (dev < 0 || dev >= MAX_DEVICES) return CHAMELEON_ERR_UNEXPECTED;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_potrf_scratch);
        if (e != cudaSuccess || !p) {
            report_cuda_error("cudaGetSymbolAddress(g_potrf_scratch)", e, __FILE__, __LINE__);
            return CHAMELEON_ERR_UNEXPECTED;
        }
        g_scratch_addr[dev] = static_cast<double *>(p);
    }
    if (!g_attr_set[dev]) {
        const cudaError_t e = cudaFuncSetAttribute(potrf_noalloc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)TILE_KERNEL_SMEM_BYTES);
        if (e != cudaSuccess) {
            report_cuda_error("cudaFuncSetAttribute(potrf_noalloc_kernel)", e, __FILE__, __LINE__);
            return CHAMELEON_ERR_UNEXPECTED;
        }
        g_attr_set[dev] = true;
    }
    *addr = g_scratch_addr[dev];
    return 0;
}
}  // namespace

}  // namespace chb

using namespace chb;

extern "C" int CUDA_dpotrf_noalloc(cham_uplo_t uplo, int n, double *A, int lda, int *d_info, void *cuda_stream) {
    if (uplo != ChamUpper && uplo != ChamLower) return -1;
    if (n < 0) return -2;
    if (lda < (n > 1 ? n : 1)) return -4;
    if (n > CHAM_B200_NOALLOC_POTRF_MAXN) {
        fprintf(stderr,
                "CUDA_dpotrf_noalloc: n = %d exceeds the fixed scratch limit of %d; use CUDA_dpotrf for larger "
                "tiles\n",
                n, CHAM_B200_NOALLOC_POTRF_MAXN);
        return CHAMELEON_ERR_INTERNAL_LIMIT;
    }
    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    if (n == 0) {
        if (d_info && cudaMemsetAsync(d_info, 0, sizeof(int), s) != cudaSuccess) return CHAMELEON_ERR_UNEXPECTED;
        return 0;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return CHAMELEON_ERR_UNEXPECTED;
    double *scratch = nullptr;
    if (int rc = noalloc_setup(dev, &scratch)) return rc;
    const View T = (uplo == ChamLower) ? View{A, 1, lda} : View{A, lda, 1};
    // a launch error left over from unrelated earlier work would otherwise be
    // reported as this launch's failure
    (void)cudaGetLastError();
    potrf_noalloc_kernel<<<1, NT_CTA, TILE_KERNEL_SMEM_BYTES, s>>>(T, n, scratch, d_info);
    CHB_LAUNCHED(1);
    return cudaGetLastError() == cudaSuccess ? CHAMELEON_SUCCESS : CHAMELEON_ERR_UNEXPECTED;
}
