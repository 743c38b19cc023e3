// wmarg_tc.cu -- Zwanzig-reweighted bimarginals as an integer one-hot GEMM
// X^T diag(w) X on the tcgen05 tensor cores (sm_100a).
//
// The weights are the fixed-point integers of mi3_weighted_marg (round(w *
// 2^s), s from the largest weight and the shared-memory kernel's chunk, so at
// most 17 bits), split into three byte planes w = w0 + 2^8 w1 + 2^16 w2.  For
// plane p the A operand holds w_p(n) at the one-hot positions of the row
// sites and the B operand the plain one-hot of the column sites, both u8;
// tcgen05.mma.kind::i8 accumulates sum_n w_p(n) [s_i=a][s_j=b] exactly in
// s32 tensor memory (at most 255 per sequence, so exact below 8.4e6
// sequences per CTA).  The epilogue recombines the planes into 64-bit
// integers, which are added with integer atomics: the result is the same
// integer sum as the shared-memory kernel's, so both give identical floats.
//
// Tile: 128 rows (the residues of floor(128/q) sites of one block) x 128
// columns (floor(128/q) sites of another) per CTA; three 128-column
// accumulators take 384 of the 512 tensor-memory columns, so one CTA per SM.
// Each K step stages the words of 128 sequences and their weight bytes,
// writes the four operand tiles (three A planes, one B) into shared memory in
// the K-major 128-byte-swizzled layout, and one thread issues 12 MMAs (3
// planes x 4 x K=32) and commits them to an mbarrier; a 2-stage ring
// overlaps generation with the MMAs.
#include "tc.cuh"

namespace mi3 {

constexpr uint32_t WT_M = 128, WT_N = 128, WT_KSTEP = 128, WT_PLANES = 3;
constexpr uint32_t WT_THREADS = 256;
constexpr uint32_t WT_A_BYTES = WT_M * 128;  // 16 KB per plane
constexpr uint32_t WT_B_BYTES = WT_N * 128;  // 16 KB
constexpr uint32_t WT_STAGE_BYTES = WT_PLANES * WT_A_BYTES + WT_B_BYTES;
constexpr uint32_t WT_MAX_WORDS = 20;  // sequence words per K step (rows + columns), q >= 4
constexpr uint32_t WT_SMEM = 1024 + 2 * WT_STAGE_BYTES + WT_MAX_WORDS * WT_KSTEP * 4 + WT_PLANES * WT_KSTEP + 64;
constexpr uint32_t WT_TMEM_COLS = 512;

// D s32, A/B unsigned 8-bit, both K-major, M=128, N=128.
constexpr uint32_t WT_IDESC = (2u << 4) | ((WT_N >> 3) << 17) | ((WT_M >> 4) << 24);

__device__ __forceinline__ void wt_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(WT_IDESC), "r"(accumulate));
}

// 0xff in every byte of w equal to the matching byte of a4, else 0.
__device__ __forceinline__ uint32_t match4(uint32_t w, uint32_t a4) {
    uint32_t x = w ^ a4;
    uint32_t nz = ((x & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | x;
    uint32_t z = ~nz & 0x80808080u;
    return (z >> 7) * 0xFFu;
}

struct WtGeom {
    uint32_t SR, SC;    // sites per row / column tile
    uint32_t nrt, nct;  // tiles per side
    uint32_t ntiles;    // (row tile, column tile) pairs holding some i < j
    uint32_t chunk, nchunks;
    uint32_t fix_chunk;  // chunk of the fixed-point scale (mi3_weighted_marg's)
};

__device__ __forceinline__ void wt_tile_coords(uint32_t t, const WtGeom &g, uint32_t &rt, uint32_t &ct) {
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

__global__ void wt_wmax(const float *__restrict__ w, uint32_t n, unsigned int *out) {
    float m = 0.0f;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) m = fmaxf(m, w[k]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m > 0.0f) atomicMax(out, __float_as_uint(m));
}

__global__ void wt_to_float(const unsigned long long *__restrict__ acc, const unsigned int *wmax_bits,
                            uint32_t fix_chunk, float *out, uint64_t n) {
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int s = fixed_shift(__uint_as_float(*wmax_bits), fix_chunk);
    out[k] = (float)ldexp((double)acc[k], -s);
}

__global__ void __launch_bounds__(WT_THREADS, 1) k_wmarg_tc(const uint32_t *__restrict__ seq, uint32_t buflen,
                                                          uint32_t nseq, const float *__restrict__ weights,
                                                          const unsigned int *__restrict__ wmax_bits,
                                                          unsigned long long *__restrict__ acc, uint32_t L,
                                                          uint32_t q, WtGeom g, int32_t *status) {
    extern __shared__ unsigned char smem_raw[];
    const uint32_t base_addr = smem_addr(smem_raw);
    const uint32_t pad = (1024u - (base_addr & 1023u)) & 1023u;
    unsigned char *sm = smem_raw + pad;  // 1024-aligned
    uint32_t *seqw = reinterpret_cast<uint32_t *>(sm + 2 * WT_STAGE_BYTES);
    unsigned char *wb = reinterpret_cast<unsigned char *>(seqw + WT_MAX_WORDS * WT_KSTEP);  // [plane][seq]
    uint64_t *mbar = reinterpret_cast<uint64_t *>(wb + WT_PLANES * WT_KSTEP);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(mbar + 2);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t tile = blockIdx.x % g.ntiles, chunk = blockIdx.x / g.ntiles;
    uint32_t rt, ct;
    wt_tile_coords(tile, g, rt, ct);
    const uint32_t i0 = rt * g.SR, j0 = ct * g.SC;
    const uint32_t nsr = min(g.SR, L - i0);
    const uint32_t nsc = j0 < L ? min(g.SC, L - j0) : 0;
    const uint32_t swords = (L - 1) / 4 + 1;
    const uint32_t wr0 = i0 / 4, nwr = (i0 + nsr - 1) / 4 - wr0 + 1;
    const uint32_t wc0 = j0 / 4, nwc = nsc ? (j0 + nsc - 1) / 4 - wc0 + 1 : 0;
    const float scale = ldexpf(1.0f, fixed_shift(__uint_as_float(*wmax_bits), g.fix_chunk));

    if (tid == 0) {
        mbar_init(&mbar[0], 1);
        mbar_init(&mbar[1], 1);
        *abort_flag = 0;
        fence_mbar_init();
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                     "r"(WT_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    // rows never generated (padding, sites past L) must read as 0
    for (uint32_t k = tid; k < 2 * WT_STAGE_BYTES / 16; k += WT_THREADS)
        reinterpret_cast<uint4 *>(sm)[k] = make_uint4(0, 0, 0, 0);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    const uint32_t nbeg = chunk * g.chunk;
    const uint32_t nend = min(nseq, nbeg + g.chunk);
    const uint32_t nk = (nend - nbeg + WT_KSTEP - 1) / WT_KSTEP;
    const uint32_t nunits = (nsr + nsc) * (WT_KSTEP / 16);
    bool ok = true;
    uint32_t nissued = 0;

    for (uint32_t ks = 0; ks < nk; ++ks) {
        const uint32_t s = ks & 1;
        if (ks >= 2) {
            if (!mbar_wait_bounded(&mbar[s], ((ks >> 1) - 1) & 1, abort_flag, WAIT_LIMIT_NS)) {
                report(status, ST_TIMEOUT_FULL);
                *abort_flag = 1;
                ok = false;
            }
        }
        __syncthreads();
        if (*abort_flag) {
            ok = false;
            break;
        }
        // stage the sequence words [word][seq] and the weight bytes [plane][seq]
        const uint32_t k0 = nbeg + ks * WT_KSTEP;
        for (uint32_t idx = tid; idx < (nwr + nwc) * WT_KSTEP; idx += WT_THREADS) {
            const uint32_t w = idx / WT_KSTEP, n = idx % WT_KSTEP;
            const uint32_t word = w < nwr ? wr0 + w : wc0 + (w - nwr);
            const uint32_t sn = k0 + n;
            seqw[w * WT_KSTEP + n] =
                (sn < nend && word < swords) ? __ldg(&seq[(size_t)word * buflen + sn]) : 0xFFFFFFFFu;
        }
        if (tid < WT_KSTEP) {
            const uint32_t sn = k0 + tid;
            const uint32_t wf = sn < nend ? __float2uint_rn(__ldg(&weights[sn]) * scale) : 0u;
            wb[tid] = wf & 0xffu;
            wb[WT_KSTEP + tid] = (wf >> 8) & 0xffu;
            wb[2 * WT_KSTEP + tid] = (wf >> 16) & 0xffu;
        }
        __syncthreads();
        unsigned char *A = sm + s * WT_STAGE_BYTES;  // 3 planes
        unsigned char *B = A + WT_PLANES * WT_A_BYTES;
        for (uint32_t u = tid; u < nunits; u += WT_THREADS) {
            const uint32_t grp = u % (WT_KSTEP / 16);
            uint32_t site = u / (WT_KSTEP / 16);
            const bool is_row = site < nsr;
            uint32_t wrow, byte;
            if (is_row) {
                const uint32_t gs = i0 + site;
                wrow = gs / 4 - wr0;
                byte = gs & 3;
            } else {
                site -= nsr;
                const uint32_t gs = j0 + site;
                wrow = nwr + gs / 4 - wc0;
                byte = gs & 3;
            }
            // residues of the site for sequences grp*16 .. +15, 4 per word
            const uint4 *src = reinterpret_cast<const uint4 *>(seqw + wrow * WT_KSTEP + grp * 16);
            uint32_t r[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                const uint4 x = src[v];
                const uint32_t lo = __byte_perm(x.x, x.y, byte | ((byte + 4) << 4));
                const uint32_t hi = __byte_perm(x.z, x.w, byte | ((byte + 4) << 4));
                r[v] = __byte_perm(lo, hi, 0x5410u);
            }
            if (is_row) {
                uint4 wp[WT_PLANES];
#pragma unroll
                for (int p = 0; p < (int)WT_PLANES; ++p)
                    wp[p] = *reinterpret_cast<const uint4 *>(wb + p * WT_KSTEP + grp * 16);
                for (uint32_t a = 0; a < q; ++a) {
                    const uint32_t a4 = a * 0x01010101u;
                    const uint32_t row = site * q + a;
                    const uint32_t m0 = match4(r[0], a4), m1 = match4(r[1], a4), m2 = match4(r[2], a4),
                                   m3 = match4(r[3], a4);
                    const uint32_t off = row * 128 + ((grp ^ (row & 7)) << 4);
#pragma unroll
                    for (int p = 0; p < (int)WT_PLANES; ++p)
                        *reinterpret_cast<uint4 *>(A + p * WT_A_BYTES + off) =
                            make_uint4(m0 & wp[p].x, m1 & wp[p].y, m2 & wp[p].z, m3 & wp[p].w);
                }
            } else {
                for (uint32_t a = 0; a < q; ++a) {
                    const uint32_t a4 = a * 0x01010101u;
                    const uint32_t row = site * q + a;
                    *reinterpret_cast<uint4 *>(B + row * 128 + ((grp ^ (row & 7)) << 4)) =
                        make_uint4(match4(r[0], a4) & 0x01010101u, match4(r[1], a4) & 0x01010101u,
                                   match4(r[2], a4) & 0x01010101u, match4(r[3], a4) & 0x01010101u);
                }
            }
        }
        fence_proxy_async_smem();
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t bbase = smem_addr(B);
#pragma unroll
            for (uint32_t p = 0; p < WT_PLANES; ++p) {
                const uint32_t abase = smem_addr(A + p * WT_A_BYTES);
#pragma unroll
                for (uint32_t kk = 0; kk < 4; ++kk)
                    wt_mma(tmem + p * WT_N, umma_desc_sw128(abase + kk * 32), umma_desc_sw128(bbase + kk * 32),
                           (ks | kk) != 0);
            }
            tc_commit(&mbar[s]);
        }
        nissued = ks + 1;
    }

    // the last commit covers every MMA issued before it; on the abort path
    // this still drains the MMAs in flight before tensor memory is freed
    if (nissued > 0) {
        const uint32_t last = nissued - 1;
        if (!mbar_wait_bounded(&mbar[last & 1], (last >> 1) & 1, nullptr, WAIT_LIMIT_NS)) {
            report(status, ST_TIMEOUT_FULL);
            *abort_flag = 1;
            ok = false;
        }
    }
    __syncthreads();
    tc_fence_after();
    if (ok && nissued == nk && nk > 0 && !*abort_flag) {
        // warp w reads lanes 32*(w%4).. (rows) and columns [64*(w/4), +64)
        const uint32_t r = 32 * (warp & 3) + lane;
        const uint32_t si = r / q, a = r % q;
        const bool rvalid = r < nsr * q;
        const uint32_t gi = i0 + si;
        const uint32_t lanebase = (32 * (warp & 3)) << 16;
        for (uint32_t c0 = 64 * (warp >> 2); c0 < 64 * (warp >> 2) + 64; c0 += 16) {
            uint32_t v0[16], v1[16], v2[16];
            tmem_ld16(tmem + lanebase + c0, v0);
            tmem_ld16(tmem + lanebase + WT_N + c0, v1);
            tmem_ld16(tmem + lanebase + 2 * WT_N + c0, v2);
            if (!rvalid) continue;
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                const uint32_t c = c0 + k;
                const uint32_t sj = c / q, b = c % q;
                const uint32_t gj = j0 + sj;
                if (c < nsc * q && gi < gj) {
                    const unsigned long long v = (unsigned long long)v0[k] + ((unsigned long long)v1[k] << 8) +
                                                 ((unsigned long long)v2[k] << 16);
                    if (v) atomicAdd(acc + pair_index(gi, gj, L) * (q * q) + a * q + b, v);
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(WT_TMEM_COLS));
}

}  // namespace mi3

using namespace mi3;

extern "C" size_t mi3_weighted_marg_tc_workspace(uint32_t L, uint32_t q) {
    return 256 + (size_t)npairs_of(L) * q * q * 8;
}

extern "C" int mi3_weighted_marg_tc(const float *weights, const uint32_t *seqmem, uint32_t buflen, uint32_t nseq,
                                    float *bimarg, uint32_t L, uint32_t q, void *workspace, size_t ws_bytes,
                                    int32_t *status, void *stream) {
    if (!weights || !seqmem || !bimarg || !workspace || !status)
        return fail(MI3_ERR_ARG, "mi3_weighted_marg_tc: null pointer");
    if (L < 2 || q < 4 || q > 32 || nseq > buflen)
        return fail(MI3_ERR_ARG, "mi3_weighted_marg_tc: bad L/q/nseq (4 <= q <= 32)");
    cudaStream_t st = as_stream(stream);
    const uint64_t nbins = npairs_of(L) * q * q;
    if (nseq == 0) {
        cudaMemsetAsync(bimarg, 0, nbins * 4, st);
        return check_launch("mi3_weighted_marg_tc: memset");
    }
    if (ws_bytes < mi3_weighted_marg_tc_workspace(L, q))
        return fail(MI3_ERR_WORKSPACE, "mi3_weighted_marg_tc: workspace too small");
    if (!aligned(workspace, 256)) return fail(MI3_ERR_ALIGN, "mi3_weighted_marg_tc: workspace must be 256B aligned");
    WtGeom g;
    g.SR = WT_M / q;
    g.SC = WT_N / q;
    g.nrt = (L + g.SR - 1) / g.SR;
    g.nct = (L + g.SC - 1) / g.SC;
    g.ntiles = 0;
    for (uint32_t r = 0; r < g.nrt; ++r) g.ntiles += g.nct - (r * g.SR) / g.SC;
    if ((g.SR + 3) / 4 + 1 + (g.SC + 3) / 4 + 1 > WT_MAX_WORDS)
        return fail(MI3_ERR_ARG, "mi3_weighted_marg_tc: q too small for the staging plan");
    // chunks of sequences: about two waves of one CTA per SM, at most 2^23
    // sequences (s32 accumulators of byte sums stay exact)
    const uint32_t want = std::max<uint32_t>(1, (148 * 2 + g.ntiles - 1) / g.ntiles);
    uint32_t chunk = (nseq + want - 1) / want;
    chunk = std::max<uint32_t>(chunk, 2048);
    chunk = std::min<uint32_t>(chunk, 1u << 23);
    chunk = (chunk + WT_KSTEP - 1) / WT_KSTEP * WT_KSTEP;
    g.chunk = chunk;
    g.nchunks = (nseq + chunk - 1) / chunk;
    g.fix_chunk = wmarg_fixed_chunk(L, q, nseq);
    uint64_t nblk = (uint64_t)g.ntiles * g.nchunks;
    if (nblk > 0x7fffffffull) return fail(MI3_ERR_ARG, "mi3_weighted_marg_tc: grid too large");
    unsigned char *ws = reinterpret_cast<unsigned char *>(workspace);
    auto *wmax = reinterpret_cast<unsigned int *>(ws);
    auto *acc = reinterpret_cast<unsigned long long *>(ws + 256);
    if (cudaMemsetAsync(ws, 0, 256 + nbins * 8, st) != cudaSuccess)
        return check_launch("mi3_weighted_marg_tc: memset");
    wt_wmax<<<296, 512, 0, st>>>(weights, nseq, wmax);
    cudaFuncSetAttribute(k_wmarg_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)WT_SMEM);
    k_wmarg_tc<<<(uint32_t)nblk, WT_THREADS, WT_SMEM, st>>>(seqmem, buflen, nseq, weights, wmax, acc, L, q, g, status);
    int rc = check_launch("mi3_weighted_marg_tc");
    if (rc) return rc;
    wt_to_float<<<(uint32_t)((nbins + 255) / 256), 256, 0, st>>>(acc, wmax, g.fix_chunk, bimarg, nbins);
    return check_launch("mi3_weighted_marg_tc: convert");
}
