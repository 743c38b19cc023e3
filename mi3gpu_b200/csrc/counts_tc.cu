// counts_tc.cu -- exact bimarginal counts as an FP8 one-hot GEMM on the
// 5th-generation tensor cores (tcgen05, sm_100a).
//
// count[(i,a),(j,b)] = sum_n X[n,(i,a)] X[n,(j,b)], X the one-hot encoding of
// the sequences (X[n,(i,a)] = 1 if s_i(n) = a).  A CTA owns one output tile
// and one chunk of sequences: 128 rows = the (site, residue) pairs of
// floor(128/q) sites of block I and 256 columns = those of floor(256/q)
// sites of block J; K runs over the chunk, 128 sequences per step.
//
// Warp roles.  Sixteen producer warps stage the step's sequence words
// ([word][seq], double-buffered) and write the one-hot tiles A (128 x 128 B)
// and B (256 x 128 B) as FP8 e4m3 (1.0 = 0x38) straight into shared memory
// in the K-major 128-byte-swizzled layout the MMA reads, into a ring of 4
// stages; each producer thread fences its writes to the async proxy and
// arrives on the stage's "full" mbarrier.  One thread of a ninth warp waits
// for it, issues four tcgen05.mma.kind::f8f6f4 (K = 32 each) into a 128 x
// 256 FP32 accumulator in tensor memory and commits them to the stage's
// "empty" mbarrier, which the producers wait on before they refill the
// stage.  After the last step the producers read the accumulator back
// (tcgen05.ld) and write the counts.  FP32 holds every integer below 2^24
// exactly, so each chunk of at most 2^24 sequences is exact; chunks are
// summed with integer atomics.
#include "tc.cuh"

namespace mi3 {

constexpr uint32_t TC_M = 128, TC_N = 256, TC_KSTEP = 128;
constexpr uint32_t TC_A_BYTES = TC_M * 128;   // 16 KB
constexpr uint32_t TC_B_BYTES = TC_N * 128;   // 32 KB
constexpr uint32_t TC_STAGE_BYTES = TC_A_BYTES + TC_B_BYTES;
constexpr uint32_t TC_MAX_WORDS = 26;         // sequence words staged per K step (rows + columns), q >= 4
constexpr uint32_t TC_STAGES = 4;
constexpr uint32_t TC_PRODUCERS = 512;        // warps 0-15: one-hot producers, then the epilogue
constexpr uint32_t TC_MMA_WARP = TC_PRODUCERS / 32;
constexpr uint32_t TC_THREADS = TC_PRODUCERS + 32;  // warp 16: TMEM allocation and the MMA-issuing thread
constexpr uint32_t TC_WORDS_BYTES = TC_MAX_WORDS * TC_KSTEP * 4;
constexpr uint32_t TC_SMEM = 1024 /*align slack*/ + TC_STAGES * TC_STAGE_BYTES + 2 * TC_WORDS_BYTES + 128;
constexpr uint32_t TC_WPT = (TC_MAX_WORDS * TC_KSTEP + TC_PRODUCERS - 1) / TC_PRODUCERS;  // staged words per producer
static_assert(TC_SMEM <= 227 * 1024, "counts_tc: shared memory");

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

// PTX prmt.b32 (default mode): byte n of the result is byte (c >> 4n) & 7 of
// {b, a} (a = bytes 0-3, b = bytes 4-7), or that byte's sign bit
// replicated when bit 3 of the nibble is set.
__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t d;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}

// 4 residue bytes -> the low 16 bits of a prmt selector, one nibble per
// byte (residue & 15); 0xFF (no sequence) becomes 0xF, whose set bit 3
// selects a sign bit -- 0 in the one-hot tables below
__device__ __forceinline__ uint32_t residue_nibbles(uint32_t r) {
    const uint32_t t = r & 0x0F0F0F0Fu;
    return prmt(t | (t >> 4), 0u, 0x0020u);
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

// true on every producer thread if pred is true on any (named barrier 1
// over the producer threads; also orders their shared-memory accesses)
__device__ __forceinline__ bool producers_any(bool pred) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, 1, %2, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)pred), "n"(TC_PRODUCERS)
        : "memory");
    return r != 0;
}

__global__ void __launch_bounds__(TC_THREADS, 1) k_counts_tc(const uint32_t *__restrict__ seq, uint32_t buflen,
                                                           uint32_t nseq, uint32_t *__restrict__ out, uint32_t L,
                                                           uint32_t q, TcGeom g, int32_t *status) {
    extern __shared__ unsigned char smem_raw[];
    const uint32_t base_addr = smem_addr(smem_raw);
    const uint32_t pad = (1024u - (base_addr & 1023u)) & 1023u;
    unsigned char *sm = smem_raw + pad;  // 1024-aligned
    uint32_t *seqw0 = reinterpret_cast<uint32_t *>(sm + TC_STAGES * TC_STAGE_BYTES);
    uint64_t *bars = reinterpret_cast<uint64_t *>(sm + TC_STAGES * TC_STAGE_BYTES + 2 * TC_WORDS_BYTES);
    uint64_t *full = bars, *empty = bars + TC_STAGES, *done = bars + 2 * TC_STAGES;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
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
        for (uint32_t s = 0; s < TC_STAGES; ++s) {
            mbar_init(&full[s], TC_PRODUCERS);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        *abort_flag = 0;
        fence_mbar_init();
    }
    if (warp == TC_MMA_WARP) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                     "r"(TC_N));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    // rows that are never generated (sites past the tile's last, padding
    // rows) must read as 0 in every stage; the generated rows are rewritten
    // in full at every step
    for (uint32_t s = 0; s < TC_STAGES; ++s) {
        uint4 *A = reinterpret_cast<uint4 *>(sm + s * TC_STAGE_BYTES);
        for (uint32_t k = nsr * q * 8 + tid; k < TC_M * 8; k += TC_THREADS) A[k] = make_uint4(0, 0, 0, 0);
        uint4 *B = reinterpret_cast<uint4 *>(sm + s * TC_STAGE_BYTES + TC_A_BYTES);
        for (uint32_t k = nsc * q * 8 + tid; k < TC_N * 8; k += TC_THREADS) B[k] = make_uint4(0, 0, 0, 0);
    }
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    const uint32_t nbeg = chunk * g.chunk;
    const uint32_t nend = min(nseq, nbeg + g.chunk);
    const uint32_t nk = (nend - nbeg + TC_KSTEP - 1) / TC_KSTEP;

    if (warp == TC_MMA_WARP) {
        // ------------------------------------------------------ MMA thread
        if (lane == 0) {
            uint32_t ks = 0;
            for (; ks < nk; ++ks) {
                const uint32_t s = ks % TC_STAGES;
                if (!mbar_wait_bounded(&full[s], (ks / TC_STAGES) & 1, abort_flag, WAIT_LIMIT_NS)) {
                    if (!*abort_flag) report(status, ST_TIMEOUT_FULL);
                    *abort_flag = 1;
                    break;
                }
                tc_fence_after();
                const uint32_t abase = smem_addr(sm + s * TC_STAGE_BYTES), bbase = abase + TC_A_BYTES;
#pragma unroll
                for (uint32_t kk = 0; kk < 4; ++kk)
                    tc_mma(tmem, umma_desc_sw128(abase + kk * 32), umma_desc_sw128(bbase + kk * 32),
                           (ks | kk) != 0);
                tc_commit(&empty[s]);
            }
            // the last commit covers every MMA issued before it
            if (ks > 0)
                tc_commit(done);
            else
                mbar_arrive(done);
        }
        __syncwarp();
    } else {
        // ------------------------------------------------------- producers
        // Staged word idx = tid + 512 j of a step is seqw[idx]: word row
        // idx / 128, sequence k0 + idx % 128.  The loads of step ks + 1 are
        // issued into registers before step ks is generated and stored to
        // shared memory at the start of step ks + 1, so their latency is
        // hidden behind one step's generation.
        const uint32_t nstaged = (nwr + nwc) * TC_KSTEP;
        uint32_t pre[TC_WPT];
        auto load_step = [&](uint32_t ks) {
            const uint32_t k0 = nbeg + ks * TC_KSTEP;
#pragma unroll
            for (uint32_t j = 0; j < TC_WPT; ++j) {
                const uint32_t idx = tid + j * TC_PRODUCERS;
                const uint32_t wd = idx / TC_KSTEP, sn = k0 + idx % TC_KSTEP;
                const uint32_t word = wd < nwr ? wr0 + wd : wc0 + (wd - nwr);
                pre[j] = (idx < nstaged && sn < nend && word < swords) ? __ldg(&seq[(size_t)word * buflen + sn])
                                                                      : 0xFFFFFFFFu;
            }
        };
        bool ok = true;
        load_step(0);
        for (uint32_t ks = 0; ks < nk; ++ks) {
            const uint32_t s = ks % TC_STAGES;
            // the MMAs of step ks - 4 must have read stage s
            const bool w = ks < TC_STAGES ||
                           mbar_wait_bounded(&empty[s], ((ks / TC_STAGES) - 1) & 1, abort_flag, WAIT_LIMIT_NS);
            // sequence words of this K step -> buffer ks & 1 ([word][seq]);
            // the barrier of step ks - 1 separated this rewrite from the
            // buffer's reads at step ks - 2
            uint32_t *seqw = seqw0 + (ks & 1) * (TC_MAX_WORDS * TC_KSTEP);
#pragma unroll
            for (uint32_t j = 0; j < TC_WPT; ++j)
                if (tid + j * TC_PRODUCERS < nstaged) seqw[tid + j * TC_PRODUCERS] = pre[j];
            if (ks + 1 < nk) load_step(ks + 1);
            if (producers_any(!w || *abort_flag)) {
                if (!w) report(status, ST_TIMEOUT_EMPTY);
                *abort_flag = 1;
                ok = false;
                break;
            }
            unsigned char *A = sm + s * TC_STAGE_BYTES;
            unsigned char *B = A + TC_A_BYTES;
            const uint32_t nunits = (nsr + nsc) * (TC_KSTEP / 16);
            for (uint32_t u = tid; u < nunits; u += TC_PRODUCERS) {
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
                // residues of site for the step's sequences 32 v + 4 grp + k
                // (v, k < 4), which go to K positions 16 grp + 4 v + k of
                // both operands (a K order shared by A and B leaves the
                // product unchanged; the 8 lanes of a quarter warp read 128
                // contiguous bytes)
                const uint32_t *src = seqw + wrow * TC_KSTEP + 4 * grp;
                uint32_t r[4];
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    uint4 x = *reinterpret_cast<const uint4 *>(src + 32 * v);
                    // byte `byte` of each of the 4 words, packed in sequence order
                    uint32_t lo = __byte_perm(x.x, x.y, byte | ((byte + 4) << 4));
                    uint32_t hi = __byte_perm(x.z, x.w, byte | ((byte + 4) << 4));
                    r[v] = __byte_perm(lo, hi, 0x5410u);
                }
                if (q <= 8) {
                    // one prmt per 4 sequences and residue: the table for a
                    // holds 0x38 at byte a and 0 elsewhere
                    uint32_t sel[4];
#pragma unroll
                    for (int v = 0; v < 4; ++v) sel[v] = residue_nibbles(r[v]);
                    for (uint32_t a = 0; a < q; ++a) {
                        const uint32_t tlo = a < 4 ? 0x38u << (8 * a) : 0u;
                        const uint32_t thi = a < 4 ? 0u : 0x38u << (8 * (a - 4));
                        const uint32_t row = site * q + a;
                        uint4 o = make_uint4(prmt(tlo, thi, sel[0]), prmt(tlo, thi, sel[1]), prmt(tlo, thi, sel[2]),
                                             prmt(tlo, thi, sel[3]));
                        *reinterpret_cast<uint4 *>(T + row * 128 + ((grp ^ (row & 7)) << 4)) = o;
                    }
                } else {
                    for (uint32_t a = 0; a < q; ++a) {
                        const uint32_t a4 = a * 0x01010101u;
                        const uint32_t row = site * q + a;
                        uint4 o = make_uint4(onehot4(r[0], a4), onehot4(r[1], a4), onehot4(r[2], a4),
                                             onehot4(r[3], a4));
                        *reinterpret_cast<uint4 *>(T + row * 128 + ((grp ^ (row & 7)) << 4)) = o;
                    }
                }
            }
            // this thread's tile writes -> visible to the tensor core
            fence_proxy_async_smem();
            mbar_arrive(&full[s]);
        }

        // ------------------------------------------------------- epilogue
        // wait for the last commit even on the abort path: the MMAs in
        // flight must drain before the tensor memory is freed
        const bool got = __all_sync(0xffffffffu, mbar_wait_bounded(done, 0, nullptr, WAIT_LIMIT_NS));
        if (!got) {
            report(status, ST_TIMEOUT_FULL);
            *abort_flag = 1;
        }
        tc_fence_after();
        if (got && ok && nk > 0 && !*abort_flag) {
            // warp w reads TMEM lanes 32*(w%4).. (rows), columns [64*(w/4), +64)
            const uint32_t r = 32 * (warp & 3) + lane;
            const uint32_t si = r / q, a = r - si * q;
            const bool rvalid = r < nsr * q;
            const uint32_t gi = i0 + si;
            const uint32_t cbeg = 64 * (warp >> 2), cend = nsc * q;
            uint32_t sj = cbeg / q, b = cbeg - sj * q;  // column (site, residue), advanced with c
#pragma unroll 1
            for (uint32_t c0 = cbeg; c0 < cbeg + 64; c0 += 16) {
                uint32_t v[16];
                tmem_ld16(tmem + ((32 * (warp & 3)) << 16) + c0, v);
#pragma unroll
                for (uint32_t k = 0; k < 16; ++k) {
                    const uint32_t gj = j0 + sj;
                    if (rvalid && c0 + k < cend && gi < gj) {
                        const uint32_t cnt = __float2uint_rn(__uint_as_float(v[k]));
                        uint32_t *dst = out + pair_index(gi, gj, L) * (q * q) + a * q + b;
                        if (g.nchunks > 1) {
                            if (cnt) atomicAdd(dst, cnt);
                        } else {
                            *dst = cnt;
                        }
                    }
                    if (++b == q) {
                        b = 0;
                        ++sj;
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == TC_MMA_WARP) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_N));
    }
}

// Tile geometry and sequence chunks of a launch (host only).  Returns false
// when the shape is outside the kernel's range.
static bool tc_plan(uint32_t L, uint32_t q, uint32_t nseq, TcGeom &g) {
    if (L < 2 || q < 4 || q > 32 || nseq == 0) return false;
    g.SR = TC_M / q;
    g.SC = TC_N / q;
    g.nrt = (L + g.SR - 1) / g.SR;
    g.nct = (L + g.SC - 1) / g.SC;
    g.ntiles = 0;
    for (uint32_t r = 0; r < g.nrt; ++r) g.ntiles += g.nct - (r * g.SR) / g.SC;
    if ((g.SR + 3) / 4 + 1 + (g.SC + 3) / 4 + 1 > TC_MAX_WORDS) return false;
    // chunks: one CTA per SM (the ring fills the shared memory).  The
    // number of chunks minimises waves x (K steps per chunk + 16, the
    // prologue and the epilogue's 32768 counts in K-step units) over 148
    // SMs, with chunks of at least 8 K steps and at most 2^24 sequences
    // (exact FP32).
    const uint32_t nks = (uint32_t)(((uint64_t)nseq + TC_KSTEP - 1) / TC_KSTEP);
    const uint32_t max_want = std::min<uint32_t>(4096, std::max<uint32_t>(1, nks / 8));
    uint32_t want = 1;
    uint64_t best = ~0ull;
    for (uint32_t w = 1; w <= max_want; ++w) {
        const uint64_t waves = ((uint64_t)g.ntiles * w + 147) / 148;
        const uint64_t cost = waves * ((nks + w - 1) / w + 16);
        if (cost < best) {
            best = cost;
            want = w;
        }
    }
    want = std::max<uint32_t>(want, (nks + (1u << 17) - 1) >> 17);
    g.chunk = (nks + want - 1) / want * TC_KSTEP;
    g.nchunks = (uint32_t)(((uint64_t)nseq + g.chunk - 1) / g.chunk);
    return true;
}

}  // namespace mi3

using namespace mi3;

extern "C" uint32_t mi3_bicounts_tc_plan(uint32_t L, uint32_t q, uint32_t nseq, uint32_t *out4) {
    TcGeom g;
    if (!tc_plan(L, q, nseq, g)) return 0;
    if (out4) {
        out4[0] = g.ntiles;
        out4[1] = g.nchunks;
        out4[2] = g.chunk;
        out4[3] = g.SR;
    }
    return 1;
}

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
    if (!tc_plan(L, q, nseq, g)) return fail(MI3_ERR_ARG, "mi3_bicounts_tc: q too small for the staging plan");
    if (g.nchunks > 1 && cudaMemsetAsync(bicount, 0, nbins * 4, st) != cudaSuccess)
        return check_launch("mi3_bicounts_tc: memset");
    cudaFuncSetAttribute(k_counts_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM);
    uint64_t nblk = (uint64_t)g.ntiles * g.nchunks;
    k_counts_tc<<<(uint32_t)nblk, TC_THREADS, TC_SMEM, st>>>(seqmem, buflen, nseq, bicount, L, q, g, status);
    return check_launch("mi3_bicounts_tc");
}
