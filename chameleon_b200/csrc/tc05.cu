// tc05.cu -- validation entry of the tcgen05 split-BF16 GEMM (tc05.cuh).
//
// CHAM_B200_Test_TC05 computes C = A B^T for A, B = 128 x K FP32 (column-major,
// ld 128) through exactly the code path the factorization uses for its
// trailing updates: split into swizzled BF16 hi/lo chunks, bulk copies into
// shared memory, tcgen05.mma into tensor memory, tcgen05.ld epilogue.  It has no
// reference counterpart; the GPU tests compare it with an FP64 product.
#include <cuda_runtime.h>

#include "core.cuh"
#include "internal.h"
#include "tc05.cuh"

namespace chb {

// X: rows x K FP32 view (rows <= 128), K % 64 == 0.  chunks: K/64 chunk pairs.
__global__ void split_rows_kernel(ViewF X, int rows, int K, uint8_t *chunks) {
    const int kc = blockIdx.x;
    uint8_t *chunk = chunks + (size_t)kc * 2 * tc05::CHUNK_BYTES;
    for (int idx = threadIdx.x; idx < 128 * tc05::BK; idx += blockDim.x) {
        const int r = idx % 128, c = idx / 128;
        const float v = (r < rows) ? *X.at(r, kc * tc05::BK + c) : 0.f;
        tc05::split_store(chunk, r, c, v);
    }
}

__global__ void __launch_bounds__(NT_CTA, 1) tc05_test_kernel(const uint8_t *a, const uint8_t *b, int nkc, float *C,
                                                              int *err) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ tc05::Smem tsm;
    // (an offset added to the __shared__ array, not a rounded integer: the
    // pointer stays visibly in shared memory, so every access through it is
    // an ld/st.shared rather than a generic load or store)
    uint8_t *stage = smem_raw + ((1024u - (unsigned)(reinterpret_cast<uintptr_t>(smem_raw) & 1023u)) & 1023u);
    tc05::init(&tsm);
    // two GEMMs in a row exercise the phase bookkeeping across tasks
    for (int rep = 0; rep < 2; ++rep) {
        const bool ok = tc05::gemm_bf16x3(
            &tsm, stage, a, b, nkc, [](int, int) {},
            [&](int r, int c0, const float *v, int) {
                if (rep == 1)
                    for (int i = 0; i < 16; ++i) C[r + (c0 + i) * 128] = v[i];
            });
        if (!ok && threadIdx.x == 0) *err = 1;
    }
    tc05::finish(&tsm);
}

}  // namespace chb

using namespace chb;

extern "C" int CHAM_B200_Test_TC05(const float *dA, const float *dB, int K, float *dC) {
    int rc = ensure_init();
    if (rc) return rc;
    if (K <= 0 || K % tc05::BK) return CHAMELEON_ERR_ILLEGAL_VALUE;
    const int nkc = K / tc05::BK;
    uint8_t *ca = nullptr, *cbuf = nullptr;
    int *err = nullptr;
    const size_t bytes = (size_t)nkc * 2 * tc05::CHUNK_BYTES;
    CHB_CUDA(cudaMalloc(&ca, bytes));
    CHB_CUDA(cudaMalloc(&cbuf, bytes));
    CHB_CUDA(cudaMalloc(&err, sizeof(int)));
    cudaStream_t s = ctx().stream;
    CHB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
    split_rows_kernel<<<nkc, 256, 0, s>>>(ViewF{const_cast<float *>(dA), 1, 128}, 128, K, ca);
    split_rows_kernel<<<nkc, 256, 0, s>>>(ViewF{const_cast<float *>(dB), 1, 128}, 128, K, cbuf);
    CHB_CUDA(cudaFuncSetAttribute(tc05_test_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, tc05::SMEM_BYTES));
    tc05_test_kernel<<<1, NT_CTA, tc05::SMEM_BYTES, s>>>(ca, cbuf, nkc, dC, err);
    CHB_LAUNCHED(3);
    CHB_CUDA(cudaGetLastError());
    int herr = 0;
    CHB_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s));
    CHB_CUDA(cudaStreamSynchronize(s));
    cudaFree(ca);
    cudaFree(cbuf);
    cudaFree(err);
    return herr ? CHAMELEON_ERR_DEVICE_TIMEOUT : 0;
}
