// counts_tc.cu -- exact bimarginal counts as an FP8 one-hot GEMM on the
// 5th-generation tensor cores (tcgen05, sm_100a).
//
// count[(i,a),(j,b)] = sum_n X[n,(i,a)] X[n,(j,b)], X the one-hot encoding of
// the sequences (X[n,(i,a)] = 1 if s_i(n) = a).  A CTA owns one output tile:
// 128 rows = the (site, residue) pairs of floor(128/q) sites of block I and
// 256 columns = those of floor(256/q) sites of block J; K runs over a chunk
// of sequences, 128 at a time.  For each K step the CTA writes the one-hot
// tiles A (128 x 128 B) and B (256 x 128 B) as FP8 e4m3 (1.0 = 0x38) straight
// into shared memory in the K-major 128-byte-swizzled layout the MMA reads,
// then one thread issues four tcgen05.mma.kind::f8f6f4 (K = 32 each) into a
// 128 x 256 FP32 accumulator in tensor memory and commits them to an
// mbarrier; a 2-stage ring lets the next tile be generated while the MMAs
// run.  FP32 holds every integer below 2^24 exactly, so each chunk of at most
// 2^24 sequences is exact; chunks are summed with integer atomics.
#include "tc.cuh"

namespace mi3 {

constexpr uint32_t TC_M = 128, TC_N = 256, TC_KSTEP = 128;
constexpr uint32_t TC_THREADS = 256;
constexpr uint32_t TC_A_BYTES = TC_M * 128;   // 16 KB
constexpr uint32_t TC_B_BYTES = TC_N * 128;   // 32 KB
constexpr uint32_t TC_STAGE_BYTES = TC_A_BYTES + TC_B_BYTES;
constexpr uint32_t TC_MAX_WORDS = 26;         // sequence words staged per K step (rows + columns), q >= 4
constexpr uint32_t TC_SMEM = 1024 /*align slack*/ + 2 * TC_STAGE_BYTES + TC_MAX_WORDS * TC_KSTEP * 4 + 64;

struct TcGeom {
    uint32_t SR, SC;       // sites per row tile / column tile
    uint32_t nrt, nct;     // tiles
    uint32_t ntiles;       // valid (row tile, column tile) pairs
    uint32_t chunk, nchunks;
};

// Instruction descriptor: D f32, A/B e4m3, both K-major, M=128, N=256.
constexpr uint32_t TC_IDESC = (1u << 4) | ((TC_N >> 3) << 17) | ((TC_M >> 4) << 24);

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(TC_IDESC), "r"(accumulate));
}

// bytes of w equal to a -> 0x38 (e4m3 1.0), others -> 0.  Per-byte zero
// test without carries between bytes: (x & 0x7f) + 0x7f sets bit 7 exactly
// when the low 7 bits are non-zero, and x's own bit 7 covers the rest.
__device__ __forceinline__ uint32_t onehot4(uint32_t w, uint32_t a4) {
    uint32_t x = w ^ a4;
    uint32_t nz = ((x & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | x;
    uint32_t z = ~nz & 0x80808080u;
    return (z >> 7) * 0x38u;
}

__device__ __forceinline__ void tile_coords(uint32_t t, const TcGeom &g, uint32_t &rt, uint32_t &ct) {
    uint32_t r = 0;
    while (true) {
        uint32_t ctmin = (r * g.SR) / g.SC;
        uint32_t cnt = g.nct - ctmin;
        if (t < cnt) {
            rt = r;
            ct = ctmin + t;
            return;
        }
        t -= cnt;
        ++r;
    }
}

__global__ void __launch_bounds__(TC_THREADS, 2) k_counts_tc(const uint32_t *__restrict__ seq, uint32_t buflen,
                                                           uint32_t nseq, uint32_t *__restrict__ out, uint32_t L,
                                                           uint32_t q, TcGeom g, int32_t *status) {
    extern __shared__ unsigned char smem_raw[];
    const uint32_t base_addr = smem_addr(smem_raw);
    const uint32_t pad = (1024u - (base_addr & 1023u)) & 1023u;
    unsigned char *sm = smem_raw + pad;  // 1024-aligned
    uint32_t *seqw = reinterpret_cast<uint32_t *>(sm + 2 * TC_STAGE_BYTES);
    uint64_t *mbar = reinterpret_cast<uint64_t *>(seqw + TC_MAX_WORDS * TC_KSTEP);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(mbar + 2);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t tile = blockIdx.x % g.ntiles, chunk = blockIdx.x / g.ntiles;
    uint32_t rt, ct;
    tile_coords(tile, g, rt, ct);
    const uint32_t i0 = rt * g.SR, j0 = ct * g.SC;
    const uint32_t nsr = min(g.SR, L - i0);              // row sites present
    const uint32_t nsc = j0 < L ? min(g.SC, L - j0) : 0; // column sites present
    const uint32_t swords = (L - 1) / 4 + 1;
    const uint32_t wr0 = i0 / 4, nwr = (i0 + nsr - 1) / 4 - wr0 + 1;
    const uint32_t wc0 = j0 / 4, nwc = nsc ? (j0 + nsc - 1) / 4 - wc0 + 1 : 0;

    if (tid == 0) {
        mbar_init(&mbar[0], 1);
        mbar_init(&mbar[1], 1);
        *abort_flag = 0;
        fence_mbar_init();
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                     "r"(TC_N));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    // zero both stages once: rows that are never generated (padding rows,
    // sites past L) must read as 0
    for (uint32_t k = tid; k < 2 * TC_STAGE_BYTES / 16; k += TC_THREADS)
        reinterpret_cast<uint4 *>(sm)[k] = make_uint4(0, 0, 0, 0);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    const uint32_t nbeg = chunk * g.chunk;
    const uint32_t nend = min(nseq, nbeg + g.chunk);
    const uint32_t nk = (nend - nbeg + TC_KSTEP - 1) / TC_KSTEP;
    const uint32_t nunits = (nsr + nsc) * (TC_KSTEP / 16);
    bool ok = true;
    uint32_t nissued = 0;  // K steps whose MMAs were issued and committed

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
        // stage the sequence words of this K step: [word][seq]
        const uint32_t k0 = nbeg + ks * TC_KSTEP;
        for (uint32_t idx = tid; idx < (nwr + nwc) * TC_KSTEP; idx += TC_THREADS) {
            uint32_t w = idx / TC_KSTEP, n = idx % TC_KSTEP;
            uint32_t word = w < nwr ? wr0 + w : wc0 + (w - nwr);
            uint32_t sn = k0 + n;
            seqw[w * TC_KSTEP + n] = (sn < nend && word < swords) ? __ldg(&seq[(size_t)word * buflen + sn]) : 0xFFFFFFFFu;
        }
        __syncthreads();
        unsigned char *A = sm + s * TC_STAGE_BYTES;
        unsigned char *B = A + TC_A_BYTES;
        for (uint32_t u = tid; u < nunits; u += TC_THREADS) {
            const uint32_t grp = u % (TC_KSTEP / 16);
            uint32_t site = u / (TC_KSTEP / 16);
            unsigned char *T;
            uint32_t wrow, byte;
            if (site < nsr) {
                T = A;
                uint32_t gs = i0 + site;
                wrow = gs / 4 - wr0;
                byte = gs & 3;
            } else {
                site -= nsr;
                T = B;
                uint32_t gs = j0 + site;
                wrow = nwr + gs / 4 - wc0;
                byte = gs & 3;
            }
            // residues of site for sequences grp*16 .. +15, packed 4 per word
            const uint4 *src = reinterpret_cast<const uint4 *>(seqw + wrow * TC_KSTEP + grp * 16);
            uint32_t r[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                uint4 x = src[v];
                // byte `byte` of each of the 4 words, packed in sequence order
                uint32_t lo = __byte_perm(x.x, x.y, byte | ((byte + 4) << 4));
                uint32_t hi = __byte_perm(x.z, x.w, byte | ((byte + 4) << 4));
                r[v] = __byte_perm(lo, hi, 0x5410u);
            }
            for (uint32_t a = 0; a < q; ++a) {
                const uint32_t a4 = a * 0x01010101u;
                const uint32_t row = site * q + a;
                uint4 o = make_uint4(onehot4(r[0], a4), onehot4(r[1], a4), onehot4(r[2], a4), onehot4(r[3], a4));
                *reinterpret_cast<uint4 *>(T + row * 128 + ((grp ^ (row & 7)) << 4)) = o;
            }
        }
        fence_proxy_async_smem();
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t abase = smem_addr(A), bbase = smem_addr(B);
#pragma unroll
            for (uint32_t kk = 0; kk < 4; ++kk)
                tc_mma(tmem, umma_desc_sw128(abase + kk * 32), umma_desc_sw128(bbase + kk * 32), (ks | kk) != 0);
            tc_commit(&mbar[s]);
        }
        nissued = ks + 1;
    }

    // wait for the last commit (it covers every MMA issued before it); on
    // the abort path this still drains the MMAs in flight before TMEM is freed
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
        // epilogue: warp w reads TMEM lanes 32*(w%4).. (rows), columns
        // [128*(w/4), +128)
        const uint32_t r = 32 * (warp & 3) + lane;
        const uint32_t si = r / q, a = r % q;
        const bool rvalid = r < nsr * q;
        const uint32_t gi = i0 + si;
        for (uint32_t c0 = 128 * (warp >> 2); c0 < 128 * (warp >> 2) + 128; c0 += 16) {
            uint32_t v[16];
            tmem_ld16(tmem + ((32 * (warp & 3)) << 16) + c0, v);
            if (!rvalid) continue;
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                const uint32_t c = c0 + k;
                const uint32_t sj = c / q, b = c % q;
                const uint32_t gj = j0 + sj;
                if (c < nsc * q && gi < gj) {
                    uint32_t cnt = __float2uint_rn(__uint_as_float(v[k]));
                    uint32_t *dst = out + pair_index(gi, gj, L) * (q * q) + a * q + b;
                    if (g.nchunks > 1) {
                        if (cnt) atomicAdd(dst, cnt);
                    } else {
                        *dst = cnt;
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_N));
}

}  // namespace mi3

using namespace mi3;

extern "C" int mi3_bicounts_tc(const uint32_t *seqmem, uint32_t buflen, uint32_t nseq, uint32_t *bicount, uint32_t L,
                               uint32_t q, int32_t *status, void *stream) {
    if (!seqmem || !bicount || !status) return fail(MI3_ERR_ARG, "mi3_bicounts_tc: null pointer");
    if (L < 2 || q < 4 || q > 32 || nseq > buflen) return fail(MI3_ERR_ARG, "mi3_bicounts_tc: bad L/q/nseq (4<=q<=32)");
    cudaStream_t st = as_stream(stream);
    const uint64_t nbins = npairs_of(L) * q * q;
    if (nseq == 0) {
        cudaMemsetAsync(bicount, 0, nbins * 4, st);
        return check_launch("mi3_bicounts_tc: memset");
    }
    TcGeom g;
    g.SR = TC_M / q;
    g.SC = TC_N / q;
    g.nrt = (L + g.SR - 1) / g.SR;
    g.nct = (L + g.SC - 1) / g.SC;
    g.ntiles = 0;
    for (uint32_t r = 0; r < g.nrt; ++r) g.ntiles += g.nct - (r * g.SR) / g.SC;
    if ((g.SR + 3) / 4 + 1 + (g.SC + 3) / 4 + 1 > TC_MAX_WORDS)
        return fail(MI3_ERR_ARG, "mi3_bicounts_tc: q too small for the staging plan");
    // chunks: at most 2^24 sequences (exact FP32), about 4 waves of 148 SMs
    uint32_t want = std::max<uint32_t>(1, (148 * 4 + g.ntiles - 1) / g.ntiles);
    uint32_t chunk = (nseq + want - 1) / want;
    chunk = std::max<uint32_t>(chunk, 4096);
    chunk = std::min<uint32_t>(chunk, 1u << 24);
    chunk = (chunk + TC_KSTEP - 1) / TC_KSTEP * TC_KSTEP;
    g.chunk = chunk;
    g.nchunks = (nseq + chunk - 1) / chunk;
    if (g.nchunks > 1 && cudaMemsetAsync(bicount, 0, nbins * 4, st) != cudaSuccess)
        return check_launch("mi3_bicounts_tc: memset");
    cudaFuncSetAttribute(k_counts_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM);
    uint64_t nblk = (uint64_t)g.ntiles * g.nchunks;
    k_counts_tc<<<(uint32_t)nblk, TC_THREADS, TC_SMEM, st>>>(seqmem, buflen, nseq, bicount, L, q, g, status);
    return check_launch("mi3_bicounts_tc");
}
