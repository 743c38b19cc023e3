// energies_tc.cu -- Potts energies as a BF16 one-hot GEMM on the tcgen05
// tensor cores (sm_100a), with a gather epilogue from tensor memory.
//
// For a tile of row sites I and column sites J, Y = X_I J_IJ is a GEMM:
// X_I is the one-hot encoding of the sequences' residues at the sites of I
// (M = 128 sequences x K = (i, a) pairs, exact in bf16) and J_IJ holds
// J_ij(a, b) for i < j (K = (i, a) x N = (j, b)), split into bf16 hi + lo
// parts so that J = hi + lo up to 2^-17 relative.  Both products accumulate
// in one FP32 accumulator in tensor memory, so
//     Y[n, (j, b)] = sum_{i in I, i < j} J_ij(s_i(n), b)
// and the sequence's energy over the tile is sum_{j in J} Y[n, (j, s_j(n))]:
// the thread owning row n reads its row of Y from tensor memory and adds
// the one column per site that its residues select.  Tile energies are
// added per sequence in 64-bit fixed point (2^-40), as mi3_energies does.
//
// A CTA owns one (row tile, column tile) pair and a range of 128-sequence
// tiles: it converts its J slice once into shared memory (hi and lo,
// K-major, 128-byte swizzle), then per sequence tile writes the one-hot A
// tile, issues 16 MMAs (2 K-blocks x 4 x K=16, hi and lo) into one of two
// tensor-memory accumulators and, while those run, reads the previous
// tile's accumulator.  Error: each coupling enters as hi + lo, within
// 2^-17 |J| of J, and Y sums at most 2 * 128 / q products in FP32.
#include <cuda_bf16.h>

#include "tc.cuh"

namespace mi3 {

constexpr uint32_t ET_M = 128, ET_N = 128, ET_K = 128;  // sequences, (j,b) columns, (i,a) rows per tile
constexpr uint32_t ET_THREADS = 128;
constexpr uint32_t ET_A_BYTES = ET_M * ET_K * 2;  // 32 KB: two K-blocks of 128 rows x 128 B
constexpr uint32_t ET_B_BYTES = ET_N * ET_K * 2;  // 32 KB each for hi and lo
constexpr uint32_t ET_MAX_WORDS = 20;             // staged sequence words per tile (rows + columns), q >= 4
constexpr uint32_t ET_SMEM = 1024 + 2 * ET_B_BYTES + 2 * ET_A_BYTES + 2 * ET_MAX_WORDS * ET_M * 4 + 64;
constexpr uint32_t ET_TMEM_COLS = 256;            // two 128-column accumulators
constexpr double ET_FIX_SCALE = 1099511627776.0;  // 2^40
constexpr double ET_FIX_INV = 1.0 / 1099511627776.0;

// D f32, A/B bf16, both K-major, M=128, N=128.
constexpr uint32_t ET_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((ET_N >> 3) << 17) | ((ET_M >> 4) << 24);

__device__ __forceinline__ void et_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(ET_IDESC), "r"(accumulate));
}

// Byte offset of element (row, k) in a K-major, 128-byte-swizzled bf16 tile
// of `rows` rows and 128 K: K-block k/64, 16-byte chunk (k%64)/8 swizzled by
// row%8, 2 bytes per element.
__device__ __forceinline__ uint32_t et_off(uint32_t rows, uint32_t row, uint32_t k) {
    const uint32_t kb = k >> 6, kin = k & 63;
    return kb * rows * 128 + row * 128 + ((((kin >> 3) ^ (row & 7)) & 7) << 4) + ((kin & 7) << 1);
}

__device__ __forceinline__ unsigned short bf16_bits(float x) {
    return __bfloat16_as_ushort(__float2bfloat16_rn(x));
}

struct EtGeom {
    uint32_t SR, SC;    // sites per row / column tile
    uint32_t nrt, nct;
    uint32_t ntiles;    // (row tile, column tile) pairs holding some i < j
    uint32_t chunk, nchunks;  // sequences per CTA (multiple of 128)
};

__device__ __forceinline__ void et_tile_coords(uint32_t t, const EtGeom &g, uint32_t &rt, uint32_t &ct) {
    uint32_t r = 0;
    while (true) {
        const uint32_t ctmin = (r * g.SR) / g.SC;
        const uint32_t cnt = g.nct - ctmin;
        if (t < cnt) {
            rt = r;
            ct = ctmin + t;
            return;
        }
        t -= cnt;
        ++r;
    }
}

__device__ __forceinline__ uint32_t et_residue(const uint32_t *words, uint32_t w, uint32_t byte, uint32_t m,
                                               uint32_t q) {
    return min((words[w * ET_M + m] >> (8 * byte)) & 0xffu, q - 1);
}

__global__ void __launch_bounds__(ET_THREADS, 1) k_energies_tc(const float *__restrict__ J,
                                                             const uint32_t *__restrict__ seq, uint32_t buflen,
                                                             uint32_t nseq, unsigned long long *__restrict__ acc,
                                                             uint32_t L, uint32_t q, EtGeom g, int32_t *status) {
    extern __shared__ unsigned char smem_raw[];
    const uint32_t base_addr = smem_addr(smem_raw);
    const uint32_t pad = (1024u - (base_addr & 1023u)) & 1023u;
    unsigned char *sm = smem_raw + pad;  // 1024-aligned
    unsigned char *Bhi = sm, *Blo = sm + ET_B_BYTES;
    unsigned char *Abuf = sm + 2 * ET_B_BYTES;  // 2 stages
    uint32_t *words = reinterpret_cast<uint32_t *>(Abuf + 2 * ET_A_BYTES);  // 2 stages of [word][seq]
    uint64_t *mbar = reinterpret_cast<uint64_t *>(words + 2 * ET_MAX_WORDS * ET_M);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(mbar + 2);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    const uint32_t tile = blockIdx.x % g.ntiles, chunk = blockIdx.x / g.ntiles;
    uint32_t rt, ct;
    et_tile_coords(tile, g, rt, ct);
    const uint32_t i0 = rt * g.SR, j0 = ct * g.SC;
    const uint32_t nsr = min(g.SR, L - i0);
    const uint32_t nsc = j0 < L ? min(g.SC, L - j0) : 0;
    const uint32_t swords = (L - 1) / 4 + 1;
    const uint32_t wr0 = i0 / 4, nwr = (i0 + nsr - 1) / 4 - wr0 + 1;
    const uint32_t wc0 = j0 / 4, nwc = nsc ? (j0 + nsc - 1) / 4 - wc0 + 1 : 0;
    const uint32_t qq = q * q;

    if (tid == 0) {
        mbar_init(&mbar[0], 1);
        mbar_init(&mbar[1], 1);
        *abort_flag = 0;
        fence_mbar_init();
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                     "r"(ET_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    // the J slice, hi and lo, once: B[(jl, b)][(il, a)] = J_ij(a, b) for
    // i < j, zero elsewhere (padding rows and columns included)
    for (uint32_t e = tid; e < ET_N * ET_K; e += ET_THREADS) {
        const uint32_t n = e / ET_K, k = e % ET_K;
        const uint32_t jl = n / q, b = n - jl * q, il = k / q, a = k - il * q;
        float v = 0.0f;
        if (jl < nsc && il < nsr && n < nsc * q && k < nsr * q) {
            const uint32_t i = i0 + il, j = j0 + jl;
            if (i < j) v = __ldg(&J[pair_index(i, j, L) * qq + a * q + b]);
        }
        const unsigned short hi = bf16_bits(v);
        const unsigned short lo = bf16_bits(v - __bfloat162float(__ushort_as_bfloat16(hi)));
        const uint32_t off = et_off(ET_N, n, k);
        *reinterpret_cast<unsigned short *>(Bhi + off) = hi;
        *reinterpret_cast<unsigned short *>(Blo + off) = lo;
    }
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    const uint32_t nbeg = chunk * g.chunk;
    const uint32_t nend = min(nseq, nbeg + g.chunk);
    const uint32_t nt = (nend - nbeg + ET_M - 1) / ET_M;
    bool ok = true;
    uint32_t nissued = 0;
    const uint32_t m = tid;  // this thread's sequence row in a tile (TMEM lane)

    // energies of the sequences of tile t from accumulator t&1
    auto epilogue = [&](uint32_t t) {
        const uint32_t s = t & 1;
        const uint32_t *w = words + s * ET_MAX_WORDS * ET_M;
        const uint32_t n = nbeg + t * ET_M + m;
        // columns this sequence selects: jl*q + s_j
        uint32_t sel[4] = {0u, 0u, 0u, 0u};
        for (uint32_t jl = 0; jl < nsc; ++jl) {
            const uint32_t gs = j0 + jl;
            const uint32_t c = jl * q + et_residue(w, nwr + gs / 4 - wc0, gs & 3, m, q);
            sel[c >> 5] |= 1u << (c & 31);
        }
        float e = 0.0f;
        const uint32_t taddr = tmem + ((32 * warp) << 16) + s * ET_N;
#pragma unroll
        for (uint32_t c0 = 0; c0 < ET_N; c0 += 16) {
            uint32_t v[16];
            tmem_ld16(taddr + c0, v);
            const uint32_t bits = (sel[c0 >> 5] >> (c0 & 31)) & 0xffffu;
#pragma unroll
            for (int k = 0; k < 16; ++k)
                if ((bits >> k) & 1u) e += __uint_as_float(v[k]);
        }
        if (n < nend) atomicAdd(&acc[n], (unsigned long long)__double2ll_rn((double)e * ET_FIX_SCALE));
    };

    for (uint32_t t = 0; t < nt; ++t) {
        const uint32_t s = t & 1;
        // accumulator and A stage s were last used by tile t-2, whose
        // epilogue ran in iteration t-1
        __syncthreads();
        if (*abort_flag) {
            ok = false;
            break;
        }
        uint32_t *w = words + s * ET_MAX_WORDS * ET_M;
        const uint32_t k0 = nbeg + t * ET_M;
        for (uint32_t idx = tid; idx < (nwr + nwc) * ET_M; idx += ET_THREADS) {
            const uint32_t wi = idx / ET_M, mm = idx % ET_M;
            const uint32_t word = wi < nwr ? wr0 + wi : wc0 + (wi - nwr);
            const uint32_t sn = k0 + mm;
            w[wi * ET_M + mm] = (sn < nend && word < swords) ? __ldg(&seq[(size_t)word * buflen + sn]) : 0u;
        }
        __syncthreads();
        // one-hot A row of sequence m: zero, then a 1.0 (bf16 0x3f80) per row site
        unsigned char *A = Abuf + s * ET_A_BYTES;
        for (uint32_t c = 0; c < ET_K / 8; ++c)
            *reinterpret_cast<uint4 *>(A + et_off(ET_M, m, 8 * c)) = make_uint4(0, 0, 0, 0);
        for (uint32_t il = 0; il < nsr; ++il) {
            const uint32_t gs = i0 + il;
            const uint32_t k = il * q + et_residue(w, gs / 4 - wr0, gs & 3, m, q);
            *reinterpret_cast<unsigned short *>(A + et_off(ET_M, m, k)) = 0x3f80u;
        }
        fence_proxy_async_smem();
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t abase = smem_addr(A), hbase = smem_addr(Bhi), lbase = smem_addr(Blo);
            uint32_t first = 1;
#pragma unroll
            for (uint32_t kb = 0; kb < 2; ++kb) {
#pragma unroll
                for (uint32_t kk = 0; kk < 4; ++kk) {
                    const uint64_t ad = umma_desc_sw128(abase + kb * ET_M * 128 + kk * 32);
                    et_mma(tmem + s * ET_N, ad, umma_desc_sw128(hbase + kb * ET_N * 128 + kk * 32), first ? 0u : 1u);
                    et_mma(tmem + s * ET_N, ad, umma_desc_sw128(lbase + kb * ET_N * 128 + kk * 32), 1u);
                    first = 0;
                }
            }
            tc_commit(&mbar[s]);
        }
        nissued = t + 1;
        // previous tile: wait for its MMAs, then read its accumulator
        if (t >= 1) {
            const uint32_t p = t - 1;
            if (!mbar_wait_bounded(&mbar[p & 1], (p >> 1) & 1, abort_flag, WAIT_LIMIT_NS)) {
                report(status, ST_TIMEOUT_FULL);
                *abort_flag = 1;
                ok = false;
            }
            tc_fence_after();
            if (ok) epilogue(p);
            tc_fence_before();
        }
    }
    // the last tile
    if (nissued > 0) {
        const uint32_t p = nissued - 1;
        if (!mbar_wait_bounded(&mbar[p & 1], (p >> 1) & 1, nullptr, WAIT_LIMIT_NS)) {
            report(status, ST_TIMEOUT_FULL);
            *abort_flag = 1;
            ok = false;
        }
        tc_fence_after();
        if (ok && !*abort_flag && nissued == nt) epilogue(p);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ET_TMEM_COLS));
}

__global__ void et_final(const unsigned long long *__restrict__ acc, float *E, uint32_t n) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) E[k] = (float)((double)(long long)acc[k] * ET_FIX_INV);
}

}  // namespace mi3

using namespace mi3;

extern "C" int mi3_energies_tc(const float *J, const uint32_t *seqmem, uint32_t buflen, uint32_t nseq,
                               float *energies, uint32_t L, uint32_t q, void *workspace, size_t ws_bytes,
                               int32_t *status, void *stream) {
    if (!J || !seqmem || !energies || !workspace || !status) return fail(MI3_ERR_ARG, "mi3_energies_tc: null pointer");
    if (L < 2 || q < 4 || q > 32 || nseq > buflen) return fail(MI3_ERR_ARG, "mi3_energies_tc: bad L/q/nseq (4<=q<=32)");
    if (nseq == 0) return MI3_OK;
    if (ws_bytes < (size_t)nseq * 8) return fail(MI3_ERR_WORKSPACE, "mi3_energies_tc: workspace too small");
    if (!aligned(workspace, 8)) return fail(MI3_ERR_ALIGN, "mi3_energies_tc: workspace alignment");
    EtGeom g;
    g.SR = ET_K / q;
    g.SC = ET_N / q;
    g.nrt = (L + g.SR - 1) / g.SR;
    g.nct = (L + g.SC - 1) / g.SC;
    g.ntiles = 0;
    for (uint32_t r = 0; r < g.nrt; ++r) g.ntiles += g.nct - (r * g.SR) / g.SC;
    if ((g.SR + 3) / 4 + 1 + (g.SC + 3) / 4 + 1 > ET_MAX_WORDS)
        return fail(MI3_ERR_ARG, "mi3_energies_tc: q too small for the staging plan");
    // sequence chunks: about two waves of one CTA per SM
    const uint32_t want = std::max<uint32_t>(1, (148 * 2 + g.ntiles - 1) / g.ntiles);
    uint32_t chunk = (nseq + want - 1) / want;
    chunk = std::max<uint32_t>(chunk, 1024);
    chunk = (chunk + ET_M - 1) / ET_M * ET_M;
    g.chunk = chunk;
    g.nchunks = (nseq + chunk - 1) / chunk;
    const uint64_t nblk = (uint64_t)g.ntiles * g.nchunks;
    if (nblk > 0x7fffffffull) return fail(MI3_ERR_ARG, "mi3_energies_tc: grid too large");
    cudaStream_t st = as_stream(stream);
    auto *acc = reinterpret_cast<unsigned long long *>(workspace);
    if (cudaMemsetAsync(acc, 0, (size_t)nseq * 8, st) != cudaSuccess) return check_launch("mi3_energies_tc: memset");
    cudaFuncSetAttribute(k_energies_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ET_SMEM);
    k_energies_tc<<<(uint32_t)nblk, ET_THREADS, ET_SMEM, st>>>(J, seqmem, buflen, nseq, acc, L, q, g, status);
    int rc = check_launch("mi3_energies_tc");
    if (rc) return rc;
    et_final<<<(nseq + 255) / 256, 256, 0, st>>>(acc, energies, nseq);
    return check_launch("mi3_energies_tc: final");
}
