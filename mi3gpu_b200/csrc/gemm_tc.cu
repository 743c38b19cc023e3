// gemm_tc.cu -- C = alpha A B^T + beta C on the tcgen05 tensor cores, BF16
// operands, FP32 accumulation and output: the dense products of the MADE
// network's training pass (forward, and the backward's input and weight
// gradients).
//
// Both operands are first packed from FP32 with arbitrary strides (so any
// transpose is a packing choice) into BF16 K-major tiles of 128 rows x 64 K
// in the 128-byte swizzled layout the MMA reads, tile (r, k) at
// ((r * Kc) + k) * 16 KB, zero outside the matrix.  One CTA computes a
// 128 x 128 block of C: a producer warp streams the A and B tiles of each
// K step into a 4-stage ring (two 1-D bulk copies on one mbarrier), one
// thread issues the MMAs (4 x K=16 per step) into a 128-column TMEM
// accumulator, and four warps write the block to C.  Waits are bounded.
#include <cuda_bf16.h>

#include <algorithm>

#include "tc.cuh"

namespace mi3 {

constexpr uint32_t GT_M = 128, GT_N = 128, GT_K = 64;
constexpr uint32_t GT_TILE = GT_M * GT_K * 2;  // 16 KB
constexpr uint32_t GT_STAGES = 4;
constexpr uint32_t GT_THREADS = 192;
constexpr uint32_t GT_SMEM = 1024 + GT_STAGES * 2 * GT_TILE + 128;
constexpr uint32_t GT_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((GT_N >> 3) << 17) | ((GT_M >> 4) << 24);

__device__ __forceinline__ uint32_t gt_sw(uint32_t row, uint32_t k) {
    return row * 128 + ((((k >> 3) ^ (row & 7)) & 7) << 4) + ((k & 7) << 1);
}

// X(r, k) = X[r * sr + k * sk] -> tile (blockIdx.y, blockIdx.x)
__global__ void __launch_bounds__(256) k_pack_bf16(const float *__restrict__ X, long long sr, long long sk,
                                                   uint32_t R, uint32_t K, uint32_t Kc, unsigned char *img) {
    __shared__ float t[GT_M][GT_K + 1];
    const uint32_t r0 = blockIdx.y * GT_M, k0 = blockIdx.x * GT_K;
    for (uint32_t e = threadIdx.x; e < GT_M * GT_K; e += 256) {
        uint32_t r, k;
        if (sk == 1) {
            r = e / GT_K;
            k = e % GT_K;
        } else {
            k = e / GT_M;
            r = e % GT_M;
        }
        const uint32_t gr = r0 + r, gk = k0 + k;
        t[r][k] = (gr < R && gk < K) ? X[(long long)gr * sr + (long long)gk * sk] : 0.0f;
    }
    __syncthreads();
    unsigned char *tile = img + ((size_t)blockIdx.y * Kc + blockIdx.x) * GT_TILE;
    for (uint32_t e = threadIdx.x; e < GT_M * (GT_K / 8); e += 256) {
        const uint32_t r = e / 8, g = e % 8;
        const float *x = &t[r][8 * g];
        uint4 w;
        w.x = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(x[0])) |
              ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(x[1])) << 16);
        w.y = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(x[2])) |
              ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(x[3])) << 16);
        w.z = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(x[4])) |
              ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(x[5])) << 16);
        w.w = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(x[6])) |
              ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(x[7])) << 16);
        *reinterpret_cast<uint4 *>(tile + gt_sw(r, 8 * g)) = w;
    }
}

__global__ void __launch_bounds__(GT_THREADS, 1)
    k_gemm_tc(const unsigned char *__restrict__ Aimg, const unsigned char *__restrict__ Bimg, uint32_t Kc, float *C,
              uint32_t M, uint32_t N, long long ldc, float alpha, float beta, int32_t *status) {
    extern __shared__ unsigned char smem_raw[];
    const uint32_t base_addr = smem_addr(smem_raw);
    unsigned char *sm = smem_raw + ((1024u - (base_addr & 1023u)) & 1023u);
    uint64_t *bars = reinterpret_cast<uint64_t *>(sm + GT_STAGES * 2 * GT_TILE);
    uint64_t *full = bars, *empty = bars + GT_STAGES, *done = bars + 2 * GT_STAGES;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    const uint32_t mt = blockIdx.x, nt = blockIdx.y;

    if (tid == 0) {
        for (uint32_t s = 0; s < GT_STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        *abort_flag = 0;
        fence_mbar_init();
    }
    if (warp == 4) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                     "r"(GT_N));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 5) {
        if ((tid & 31) == 0) {
            uint32_t kc = 0;
            for (; kc < Kc; ++kc) {
                const uint32_t s = kc % GT_STAGES, round = kc / GT_STAGES;
                if (round > 0 && !mbar_wait_bounded(&empty[s], (round - 1) & 1, abort_flag, WAIT_LIMIT_NS)) {
                    report(status, ST_TIMEOUT_EMPTY);
                    *abort_flag = 1;
                    break;
                }
                unsigned char *slot = sm + s * 2 * GT_TILE;
                mbar_arrive_expect_tx(&full[s], 2 * GT_TILE);
                bulk_g2s(slot, Aimg + ((size_t)mt * Kc + kc) * GT_TILE, GT_TILE, &full[s]);
                bulk_g2s(slot + GT_TILE, Bimg + ((size_t)nt * Kc + kc) * GT_TILE, GT_TILE, &full[s]);
            }
            for (uint32_t k = 0; k < GT_STAGES && k < kc; ++k) {
                const uint32_t j = kc - 1 - k;
                mbar_wait_bounded(&full[j % GT_STAGES], (j / GT_STAGES) & 1, nullptr, WAIT_LIMIT_NS);
            }
        }
    } else if (warp == 4) {
        if ((tid & 31) == 0) {
            const uint32_t base = smem_addr(sm);
            for (uint32_t kc = 0; kc < Kc; ++kc) {
                const uint32_t s = kc % GT_STAGES;
                if (!mbar_wait_bounded(&full[s], (kc / GT_STAGES) & 1, abort_flag, WAIT_LIMIT_NS)) {
                    report(status, ST_TIMEOUT_FULL);
                    *abort_flag = 1;
                    break;
                }
                tc_fence_after();
                const uint32_t a = base + s * 2 * GT_TILE, b = a + GT_TILE;
#pragma unroll
                for (uint32_t kk = 0; kk < GT_K / 16; ++kk) {
                    const uint32_t acc = (kc | kk) ? 1u : 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                        "l"(umma_desc_sw128(a + kk * 32)), "l"(umma_desc_sw128(b + kk * 32)), "r"(GT_IDESC),
                        "r"(acc));
                }
                tc_commit(&empty[s]);
            }
            tc_commit(done);
        }
    } else {
        // epilogue: thread = row of the block
        const bool got = __all_sync(0xffffffffu, mbar_wait_bounded(done, 0, abort_flag, WAIT_LIMIT_NS));
        if (!got) {
            report(status, ST_TIMEOUT_FULL);
            *abort_flag = 1;
        } else {
            tc_fence_after();
            const uint32_t row = mt * GT_M + 32 * warp + (tid & 31);
            const uint32_t taddr = tmem + ((32 * warp) << 16);
#pragma unroll 1
            for (uint32_t c0 = 0; c0 < GT_N; c0 += 16) {
                uint32_t v[16];
                tmem_ld16(taddr + c0, v);
                if (row < M) {
                    float *crow = C + (long long)row * ldc;
#pragma unroll
                    for (uint32_t k = 0; k < 16; ++k) {
                        const uint32_t col = nt * GT_N + c0 + k;
                        if (col < N) {
                            const float x = alpha * __uint_as_float(v[k]);
                            crow[col] = beta != 0.0f ? x + beta * crow[col] : x;
                        }
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 4) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(GT_N));
    }
}

static inline uint32_t gt_cdiv(uint64_t a, uint32_t b) { return (uint32_t)((a + b - 1) / b); }

}  // namespace mi3

using namespace mi3;

extern "C" uint64_t mi3_gemm_bf16_workspace(uint32_t M, uint32_t N, uint32_t K) {
    const uint64_t kc = gt_cdiv(K, GT_K);
    return ((uint64_t)gt_cdiv(M, GT_M) + gt_cdiv(N, GT_N)) * kc * GT_TILE;
}

extern "C" int mi3_gemm_bf16(uint32_t M, uint32_t N, uint32_t K, const float *A, int64_t sam, int64_t sak,
                             const float *B, int64_t sbk, int64_t sbn, float *C, int64_t ldc, float alpha, float beta,
                             void *workspace, uint64_t ws_bytes, int32_t *status, void *stream) {
    if (!A || !B || !C || !workspace || !status) return fail(MI3_ERR_ARG, "mi3_gemm_bf16: null pointer");
    if (M == 0 || N == 0 || K == 0) return fail(MI3_ERR_ARG, "mi3_gemm_bf16: empty matrix");
    if (ws_bytes < mi3_gemm_bf16_workspace(M, N, K)) return fail(MI3_ERR_WORKSPACE, "mi3_gemm_bf16: workspace too small");
    if (!aligned(workspace, 1024)) return fail(MI3_ERR_ALIGN, "mi3_gemm_bf16: workspace alignment (1024 B)");
    const uint32_t Mt = gt_cdiv(M, GT_M), Nt = gt_cdiv(N, GT_N), Kc = gt_cdiv(K, GT_K);
    if (Mt > 65535 || Nt > 65535) return fail(MI3_ERR_ARG, "mi3_gemm_bf16: matrix too large");
    cudaStream_t st = as_stream(stream);
    unsigned char *Aimg = reinterpret_cast<unsigned char *>(workspace);
    unsigned char *Bimg = Aimg + (size_t)Mt * Kc * GT_TILE;
    k_pack_bf16<<<dim3(Kc, Mt), 256, 0, st>>>(A, sam, sak, M, K, Kc, Aimg);
    int rc = check_launch("mi3_gemm_bf16: pack A");
    if (rc) return rc;
    k_pack_bf16<<<dim3(Kc, Nt), 256, 0, st>>>(B, sbn, sbk, N, K, Kc, Bimg);
    rc = check_launch("mi3_gemm_bf16: pack B");
    if (rc) return rc;
    cudaFuncSetAttribute(k_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GT_SMEM);
    k_gemm_tc<<<dim3(Mt, Nt), GT_THREADS, GT_SMEM, st>>>(Aimg, Bimg, Kc, C, M, N, ldc, alpha, beta, status);
    return check_launch("mi3_gemm_bf16");
}
