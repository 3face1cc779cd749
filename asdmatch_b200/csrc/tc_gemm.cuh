// BF16 x BF16 -> FP32 tile GEMM on the 5th-generation tensor cores (tcgen05).
//
//   D[m][n] = sum_k A(m, k) * B(n, k)      one 128 x 128 output tile per CTA
//
// A and B are read from global memory through caller-supplied strides (so a
// transposed operand costs nothing extra), staged 64 K-elements at a time into
// shared memory in the canonical K-major, no-swizzle core-matrix layout
// (8 rows x 16 bytes per core matrix), and multiplied by tcgen05.mma issued
// from one thread, M=128 N=128 K=16 per instruction, accumulating in tensor
// memory.  tcgen05.commit arrives on an mbarrier that every thread waits on
// (bounded) before the shared buffers are refilled or the accumulator is read
// back with tcgen05.ld.  128 threads (4 warps): warp w owns TMEM lanes
// 32w..32w+31, i.e. output rows 32w..32w+31 of the tile.
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

namespace asdm {
namespace tc {

constexpr int kTileM = 128, kTileN = 128, kChunkK = 64;
constexpr int kThreads = 128;
constexpr uint32_t kTmemCols = 128;
constexpr uint32_t kWaitSpins = 1u << 22;
// shared memory: A chunk + B chunk (16 KB each), mbarrier, TMEM address.
// Requested at 72 KB so that at most 3 CTAs share an SM: 3 x 128 TMEM
// columns never exceed the SM's 512, so tcgen05.alloc never has to wait.
constexpr int kSmemUsed = 2 * kTileM * kChunkK * 2 + 64;
constexpr int kSmemBytes = 72 * 1024;

// Operand view: element (r, k) at ptr[r * sr + k * sk]; rows >= rows_valid
// and k >= K read as zero.
struct Operand {
    const __nv_bfloat16 *ptr;
    long long sr, sk;
    int rows_valid;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// tcgen05 shared-memory matrix descriptor, SWIZZLE_NONE, version 1.
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFF) >> 4);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= 1ull << 46;  // descriptor version for sm_100
    return d;           // base offset 0, absolute-LBO mode off, layout type 0 (no swizzle)
}

// Instruction descriptor, kind::f16: D=F32, A=B=BF16, both K-major, M=128, N=128.
__host__ __device__ constexpr uint32_t idesc_bf16_f32() {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kTileN >> 3) << 17) | ((uint32_t)(kTileM >> 4) << 24);
}

// Stage rows [r0, r0+128) x k [k0, k0+64) of an operand into the core-matrix
// layout: core (row group g, k group c) at byte ((c * 16) + g) * 128, row r of
// the group at +16 r, 8 bf16 per row.
__device__ __forceinline__ void stage(__nv_bfloat16 *dst, const Operand &op, int r0, int k0, int K) {
    for (int i = threadIdx.x; i < kTileM * kChunkK; i += kThreads) {
        const int r = i / kChunkK, k = i % kChunkK;
        const int gr = r0 + r, gk = k0 + k;
        __nv_bfloat16 v = __float2bfloat16(0.f);
        if (gr < op.rows_valid && gk < K) v = op.ptr[(long long)gr * op.sr + (long long)gk * op.sk];
        const int off = (((k >> 3) * (kTileM / 8) + (r >> 3)) * 64) + ((r & 7) * 8) + (k & 7);  // in elements
        dst[off] = v;
    }
}

// Computes one 128x128 tile into acc_out (fp32, row-major with stride ldc),
// rows >= m_valid / cols >= n_valid not written.  `err` gets 1 if a wait on
// the tensor cores ran out of its bound (the tile is then not written).
__device__ void gemm_tile(const Operand &A, const Operand &B, int K, int m0, int n0, float *C, long long ldc,
                          int m_valid, int n_valid, const float *bias, bool relu, unsigned int *err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __nv_bfloat16 *sA = reinterpret_cast<__nv_bfloat16 *>(smem);
    __nv_bfloat16 *sB = sA + kTileM * kChunkK;
    uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + 2 * kTileM * kChunkK * 2);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(mbar + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)));
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = *tmem_slot;

    bool ok = true;
    uint32_t phase = 0;
    const uint32_t idesc = idesc_bf16_f32();
    for (int k0 = 0; k0 < K && ok; k0 += kChunkK) {
        stage(sA, A, m0, k0, K);
        stage(sB, B, n0, k0, K);
        // make the generic-proxy smem writes visible to the tensor cores
        asm volatile("fence.proxy.async.shared::cta;");
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            for (int s = 0; s < kChunkK / 16; ++s) {
                // K slice s: k groups 2s, 2s+1 -> byte offset 2s * 16 * 128
                const uint64_t da = make_desc(smem_u32(sA) + s * 2 * (kTileM / 8) * 128, (kTileM / 8) * 128, 128);
                const uint64_t db = make_desc(smem_u32(sB) + s * 2 * (kTileN / 8) * 128, (kTileN / 8) * 128, 128);
                const uint32_t accumulate = (k0 > 0 || s > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
                    :
                    : "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                smem_u32(mbar)));
        }
        // every thread waits for the MMAs before the buffers are reused
        uint32_t done = 0;
        for (uint32_t it = 0; it < kWaitSpins && !done; ++it) {
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                "selp.u32 %0, 1, 0, p;\n\t}\n"
                : "=r"(done)
                : "r"(smem_u32(mbar)), "r"(phase));
        }
        ok = __syncthreads_and(done != 0);
        phase ^= 1;
    }
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (ok) {
        const int row = m0 + warp * 32 + lane;
        for (int c = 0; c < kTileN; c += 8) {
            uint32_t r[8];
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
                         : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                         : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c));
            asm volatile("tcgen05.wait::ld.sync.aligned;");
            if (row < m_valid) {
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int col = n0 + c + j;
                    if (col < n_valid) {
                        float v = __uint_as_float(r[j]);
                        if (bias) v += bias[col];
                        if (relu) v = fmaxf(v, 0.f);
                        C[(long long)row * ldc + col] = v;
                    }
                }
            }
        }
    } else {
        // a wait ran out: give any MMA still in flight one more bounded wait
        // before the accumulator's tensor memory is released
        uint32_t done = 0;
        for (uint32_t it = 0; it < kWaitSpins && !done; ++it) {
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                "selp.u32 %0, 1, 0, p;\n\t}\n"
                : "=r"(done)
                : "r"(smem_u32(mbar)), "r"(phase ^ 1u));
        }
        if (threadIdx.x == 0) atomicExch(err, 1u);
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

// grid (ceil(M/128), ceil(N/128)); dynamic shared memory kSmemBytes.
__global__ void __launch_bounds__(kThreads) gemm_kernel(Operand A, Operand B, int M, int N, int K, float *C, long long ldc,
                                                        const float *bias, int relu, unsigned int *err) {
    gemm_tile(A, B, K, blockIdx.x * kTileM, blockIdx.y * kTileN, C, ldc, M, N, bias, relu != 0, err);
}

}  // namespace tc
}  // namespace asdm
