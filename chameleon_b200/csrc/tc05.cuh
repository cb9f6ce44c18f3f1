// tc05.cuh -- 5th-generation tensor-core (tcgen05 / TMEM) building blocks for
// the FP32 trailing update of the split-precision factorization.
//
//   C(128 x 128, FP32) -= A(128 x K) * B(128 x K)^T,  A, B = hi + lo in BF16
//
// computed as hi*hi + hi*lo + lo*hi on tcgen05.mma kind::f16 (BF16 inputs,
// FP32 accumulation in tensor memory).  Operands are stored once, by the panel
// solve that produces them, as "split chunks": for each 128-row block and each
// 64-wide k chunk, 16 KB of hi followed by 16 KB of lo, every row 128 bytes,
// already in the K-major 128-byte-swizzled canonical layout of the tensor core
// (16-byte column group g of row r stored at group g ^ (r & 7)).  A chunk is
// therefore one contiguous bulk copy (cp.async.bulk, TMA engine) into a
// 1024-byte aligned shared-memory stage, and the MMA reads it through a shared
// memory descriptor (SWIZZLE_128B, SBO = 1024 B).
//
// Roles inside the 256-thread CTA: thread 0 issues the bulk copies, thread 32
// issues the MMAs, all 8 warps run the epilogue (TMEM lanes 32*(warp%4)..+31,
// warps 0-3 columns 0-63, warps 4-7 columns 64-127).  Every mbarrier wait is
// bounded; on expiry the task records an error and returns.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace chb {
namespace tc05 {

constexpr int BM = 128, BN = 128, BK = 64;   // output block, k chunk
constexpr int CHUNK_BYTES = 128 * BK * 2;     // one operand half (hi or lo): 16 KB
constexpr int STAGES = 3;
constexpr int STAGE_BYTES = 4 * CHUNK_BYTES;  // A hi, A lo, B hi, B lo
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 /*alignment*/ + 256 /*barriers*/;
constexpr int TMEM_COLS = 256;   // accumulator (columns 0-127) + staged C (128-255)
constexpr unsigned long long WAIT_NS = 2000000000ull;   // bound of one mbarrier wait (2 s)

// Byte offset of element (r, c) (r < 128, c < 64) inside one swizzled chunk half.
__host__ __device__ __forceinline__ int swz_off(int r, int c) {
    return r * 128 + ((((c >> 3) ^ (r & 7)) & 7) << 4) + ((c & 7) << 1);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    return t;
}
// Bounded wait for phase `parity` to complete; false when WAIT_NS ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
    unsigned long long t0 = 0;
    for (unsigned i = 0;; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if ((i & 255) == 0) {
            const unsigned long long t = now_ns();
            if (i == 0) t0 = t;
            else if (t - t0 > WAIT_NS) return false;
        }
    }
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async;\n" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

// Shared-memory matrix descriptor: K-major, SWIZZLE_128B, SBO = 1024 B
// (8-row groups), LBO unused (1), version 1.
__device__ __forceinline__ uint64_t sdesc(const void *smem_tile) {
    const uint64_t a = (smem_u32(smem_tile) >> 4) & 0x3FFFull;
    return a | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}
// Instruction descriptor, kind::f16: D = F32, A = B = BF16, both K-major,
// N = 128, M = 128.
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                           ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(IDESC), "r"(accumulate));
}
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                     smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
        "[%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Warp-collective store of 16 consecutive 32-bit columns of this warp's TMEM
// lanes (v[i] -> column taddr + i of the thread's lane); complete with tmem_wait_st.
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const float *v) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};\n" ::"r"(
            taddr),
        "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
        "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
        "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])), "r"(__float_as_uint(v[8])),
        "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
        "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])),
        "r"(__float_as_uint(v[15]))
        : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory"); }

// One warp allocates TMEM_COLS columns; the address lands in *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t *slot) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(slot)),
                 "r"((uint32_t)TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"((uint32_t)TMEM_COLS)
                 : "memory");
}

// Per-CTA state kept in shared memory across tasks.  Barriers are initialized
// once per CTA (init()); the phase of each use follows from the running count
// of k chunks (`chunks`) and of finished GEMMs (`gemms`), so no barrier is ever
// re-initialized while an arrival could still be in flight.
struct Smem {
    uint64_t full[STAGES];
    uint64_t empty[STAGES];
    uint64_t accdone;
    uint32_t tmem;
    uint32_t chunks;
    uint32_t gemms;
    int err;
};

// Kernel prologue (all threads): barriers + TMEM allocation by warp 0.
__device__ inline void init(Smem *sm) {
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&sm->full[s], 1);
            mbar_init(&sm->empty[s], 1);
        }
        mbar_init(&sm->accdone, 1);
        sm->chunks = 0;
        sm->gemms = 0;
        sm->err = 0;
        fence_mbar_init();
        fence_proxy_async();
    }
    if ((threadIdx.x >> 5) == 0) tmem_alloc(&sm->tmem);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
}

// Kernel epilogue (all threads): release TMEM (warp 0).
__device__ inline void finish(Smem *sm) {
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    if ((threadIdx.x >> 5) == 0) tmem_free(sm->tmem);
}

// Writes the split (hi, lo) of v at (r, c) of one chunk pair.
__device__ __forceinline__ void split_store(uint8_t *chunk, int r, int c, float v) {
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    const __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
    const int off = swz_off(r, c);
    *reinterpret_cast<__nv_bfloat16 *>(chunk + off) = h;
    *reinterpret_cast<__nv_bfloat16 *>(chunk + CHUNK_BYTES + off) = l;
}

// Eight consecutive elements (r, c0 .. c0+7), c0 % 8 == 0, of one row: the
// same hi / lo values as eight split_store calls, written as one 16-byte
// group into each half.
__device__ __forceinline__ void split_store8(uint8_t *chunk, int r, int c0, const float (&v)[8]) {
    uint4 hi, lo;
    split_bf16(v[0], v[1], hi.x, lo.x);
    split_bf16(v[2], v[3], hi.y, lo.y);
    split_bf16(v[4], v[5], hi.z, lo.z);
    split_bf16(v[6], v[7], hi.w, lo.w);
    const int off = swz_off(r, c0);
    *reinterpret_cast<uint4 *>(chunk + off) = hi;
    *reinterpret_cast<uint4 *>(chunk + CHUNK_BYTES + off) = lo;
}

// acc = A * B^T over nkc chunks, A chunks at a_chunks[kc], B at b_chunks[kc]
// (each chunk = hi 16 KB + lo 16 KB, consecutive chunks 32 KB apart), then
// f(row, col0, v[16]) for accumulator row `row`, columns col0..col0+15, by the
// owning thread.  pre(row, col0) runs first, once per thread for the 64
// columns it owns (col0 = its column half), so that the epilogue's global reads
// can be issued before the accumulator is read; epilogue then gets
// (row, col0 + 16 p, v, p) for p = 0..3.  Call with all 256 threads.  Returns
// false on a wait timeout.  idle() runs on thread 64 (otherwise idle until the
// accumulator is ready) while the copies and MMAs run.
struct NoIdle {
    __device__ void operator()() const {}
};
template <class P, class F, class I = NoIdle>
__device__ bool gemm_bf16x3(Smem *sm, uint8_t *stage_base, const uint8_t *a_chunks, const uint8_t *b_chunks,
                            int nkc, P &&pre, F &&epilogue, I &&idle = I{}) {
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t base = sm->chunks;      // k chunks issued by this CTA before this GEMM
    const uint32_t gnum = sm->gemms;       // GEMMs finished by this CTA before this one
    __syncthreads();
    if (tid == 0) {
        // producer: bulk copies of the four chunk halves of each k chunk
        fence_proxy_async();   // generic-proxy writes of the operands (other SMs) -> async-proxy reads
        for (int kc = 0; kc < nkc; ++kc) {
            const uint32_t g = base + kc;
            const int s = g % STAGES;
            if (g >= STAGES && !mbar_wait(&sm->empty[s], ((g / STAGES) - 1) & 1)) {
                sm->err = 1;
                break;
            }
            uint8_t *st = stage_base + s * STAGE_BYTES;
            mbar_expect_tx(&sm->full[s], STAGE_BYTES);
            bulk_g2s(st, a_chunks + (size_t)kc * 2 * CHUNK_BYTES, 2 * CHUNK_BYTES, &sm->full[s]);
            bulk_g2s(st + 2 * CHUNK_BYTES, b_chunks + (size_t)kc * 2 * CHUNK_BYTES, 2 * CHUNK_BYTES, &sm->full[s]);
        }
    } else if (tid == 32) {
        // MMA issuer
        for (int kc = 0; kc < nkc; ++kc) {
            const uint32_t g = base + kc;
            const int s = g % STAGES;
            if (!mbar_wait(&sm->full[s], (g / STAGES) & 1)) {
                sm->err = 1;
                break;
            }
            fence_after_sync();
            uint8_t *st = stage_base + s * STAGE_BYTES;
            const uint64_t ahi = sdesc(st), alo = sdesc(st + CHUNK_BYTES);
            const uint64_t bhi = sdesc(st + 2 * CHUNK_BYTES), blo = sdesc(st + 3 * CHUNK_BYTES);
#pragma unroll
            for (int k16 = 0; k16 < BK / 16; ++k16) {
                const uint64_t dk = (uint64_t)(k16 * 32) >> 4;   // +32 bytes inside the swizzle atom
                const uint32_t acc0 = (kc > 0 || k16 > 0) ? 1u : 0u;
                mma_bf16(sm->tmem, alo + dk, bhi + dk, acc0);
                mma_bf16(sm->tmem, ahi + dk, blo + dk, 1u);
                mma_bf16(sm->tmem, ahi + dk, bhi + dk, 1u);
            }
            mma_commit(&sm->empty[s]);   // stage free once these MMAs have read it
        }
        mma_commit(&sm->accdone);
    } else if (tid == 64) {
        idle();
    }
    // epilogue: everyone waits for the accumulator
    bool ok = mbar_wait(&sm->accdone, gnum & 1);
    __syncthreads();
    if (sm->err) ok = false;
    if (ok) {
        fence_after_sync();
        const int q = warp & 3;                 // TMEM lane quarter of this warp
        const int cbase = (warp >> 2) * 64;     // column half
        const int row = q * 32 + lane;
        pre(row, cbase);
#pragma unroll
        for (int cc = 0; cc < 64; cc += 16) {
            float v[16];
            tmem_ld16(sm->tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(cbase + cc), v);
            epilogue(row, cbase + cc, (const float *)v, cc >> 4);
        }
    }
    fence_before_sync();
    __syncthreads();
    if (tid == 0) {
        sm->chunks = base + nkc;
        sm->gemms = gnum + 1;
    }
    __syncthreads();
    return ok;
}

// C -= A * B^T for one 128 x 128 block of the executor's trailing update over
// the k chunks of `ntiles` panels (nkc_tile chunks each; the panels' chunks
// are tile_stride bytes apart), accumulated in one TMEM accumulator; operands
// and roles as in gemm_bf16x3 (thread 0 copies, thread 32 MMAs, idle() on
// thread 64).  The old values of C are staged in TMEM (columns
// 128-255) by warps 4-7 while the copies and MMAs run: each of those warps
// owns one TMEM lane quarter (32 rows), reads its 128 columns 32 at a time
// and stores them with tcgen05.st, so no value stays in registers across the
// roles and the producer and MMA threads never wait on C.  The epilogue (all
// 8 warps, 64 columns each) then reads accumulator and old value from TMEM.
// load(row, col): old value (0 where nothing is written); store(row, col, v):
// writes where the task owns the element.  ph (tracing, may be null): clock
// cycles from the start to the staging of C being done (ph[0], warp 4), to the
// accumulator being ready (ph[1]) and to the end (ph[2]).  Call with all 256
// threads.  Returns false on a wait timeout.
template <class L, class S, class I>
__device__ bool gemm_bf16x3_sub(Smem *sm, uint8_t *stage_base, const uint8_t *a_chunks, const uint8_t *b_chunks,
                                int nkc_tile, int ntiles, size_t tile_stride, L &&load, S &&store, I &&idle,
                                unsigned *ph = nullptr) {
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t base = sm->chunks;   // k chunks issued by this CTA before this GEMM
    const uint32_t gnum = sm->gemms;    // GEMMs finished by this CTA before this one
    const int nkc = nkc_tile * ntiles;  // k chunks of the whole group
    __syncthreads();
    const long long c_start = ph ? clock64() : 0;
    if (tid == 0) {
        fence_proxy_async();   // generic-proxy writes of the operands (other SMs) -> async-proxy reads
        int kt = 0, kk = 0;    // panel of the group, chunk within the panel
        for (int kc = 0; kc < nkc; ++kc) {
            const uint32_t g = base + kc;
            const int s = g % STAGES;
            if (g >= STAGES && !mbar_wait(&sm->empty[s], ((g / STAGES) - 1) & 1)) {
                sm->err = 1;
                break;
            }
            uint8_t *st = stage_base + s * STAGE_BYTES;
            const size_t off = (size_t)kt * tile_stride + (size_t)kk * 2 * CHUNK_BYTES;
            mbar_expect_tx(&sm->full[s], STAGE_BYTES);
            bulk_g2s(st, a_chunks + off, 2 * CHUNK_BYTES, &sm->full[s]);
            bulk_g2s(st + 2 * CHUNK_BYTES, b_chunks + off, 2 * CHUNK_BYTES, &sm->full[s]);
            if (++kk == nkc_tile) {
                kk = 0;
                ++kt;
            }
        }
    } else if (tid == 32) {
        for (int kc = 0; kc < nkc; ++kc) {
            const uint32_t g = base + kc;
            const int s = g % STAGES;
            if (!mbar_wait(&sm->full[s], (g / STAGES) & 1)) {
                sm->err = 1;
                break;
            }
            fence_after_sync();
            uint8_t *st = stage_base + s * STAGE_BYTES;
            const uint64_t ahi = sdesc(st), alo = sdesc(st + CHUNK_BYTES);
            const uint64_t bhi = sdesc(st + 2 * CHUNK_BYTES), blo = sdesc(st + 3 * CHUNK_BYTES);
#pragma unroll
            for (int k16 = 0; k16 < BK / 16; ++k16) {
                const uint64_t dk = (uint64_t)(k16 * 32) >> 4;   // +32 bytes inside the swizzle atom
                const uint32_t acc0 = (kc > 0 || k16 > 0) ? 1u : 0u;
                mma_bf16(sm->tmem, alo + dk, bhi + dk, acc0);
                mma_bf16(sm->tmem, ahi + dk, blo + dk, 1u);
                mma_bf16(sm->tmem, ahi + dk, bhi + dk, 1u);
            }
            mma_commit(&sm->empty[s]);   // stage free once these MMAs have read it
        }
        mma_commit(&sm->accdone);
    } else if (tid == 64) {
        idle();
    } else if (warp >= 4) {
        const int q = warp & 3, row = q * 32 + lane;
        const uint32_t tc = sm->tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)BN;
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            float v[32];
#pragma unroll
            for (int i = 0; i < 32; ++i) v[i] = load(row, h * 32 + i);
#pragma unroll
            for (int j = 0; j < 2; ++j) tmem_st16(tc + (uint32_t)(h * 32 + j * 16), v + j * 16);
        }
        tmem_wait_st();
        if (ph && tid == 128) ph[0] += (unsigned)(clock64() - c_start);
    }
    // epilogue: everyone waits for the accumulator
    bool ok = mbar_wait(&sm->accdone, gnum & 1);
    if (ph && tid == 0) ph[1] += (unsigned)(clock64() - c_start);
    fence_before_sync();   // the staging warps' TMEM stores before the other warps' reads
    __syncthreads();
    if (sm->err) ok = false;
    if (ok) {
        fence_after_sync();
        const int q = warp & 3;                 // TMEM lane quarter of this warp
        const int cbase = (warp >> 2) * 64;     // column half
        const int row = q * 32 + lane;
        const uint32_t tl = sm->tmem + ((uint32_t)(q * 32) << 16);
#pragma unroll
        for (int cc = 0; cc < 64; cc += 16) {
            float v[16], o[16];
            tmem_ld16(tl + (uint32_t)(cbase + cc), v);
            tmem_ld16(tl + (uint32_t)(BN + cbase + cc), o);
#pragma unroll
            for (int i = 0; i < 16; ++i) store(row, cbase + cc + i, o[i] - v[i]);
        }
    }
    fence_before_sync();
    __syncthreads();
    if (tid == 0) {
        sm->chunks = base + nkc;
        sm->gemms = gnum + 1;
        if (ph) ph[2] += (unsigned)(clock64() - c_start);
    }
    __syncthreads();
    return ok;
}

}  // namespace tc05
}  // namespace chb
