// mcmc_skew.cu -- Metropolis sampler with bank-conflict-free coupling gathers.
//
// The reference's DeltaEnergy (mcmc.cl:360-413) sums, for each walker and in
// site order m = 0..L-1, the difference J[pos,m](mut, s_m) - J[pos,m](cur, s_m).
// When all 32 lanes of a warp read their walkers' couplings at the SAME site m
// (k_metropolis in mcmc.cu), the 32 addresses fall on random banks of one q*q
// block: about 3.1 shared-memory wavefronts per gather, and the shared-memory
// pipe is the bound.  Here lane w of a warp runs w sites behind lane 0: at
// loop iteration t it adds the term of site m = t - w.  The coupling chunk in
// shared memory is stored cell-major ([a*q + b][site column]), so the 32 lanes
// of one gather read 32 different site columns -- 32 different banks, one
// wavefront -- while every walker still adds its terms in site order with the
// same float operations: the trajectories are bit-identical to k_metropolis
// and to the oracle's restatement of the reference.
//
// Lane w keeps its walker's sequence in registers, 5-bit residues, 6 per
// 32-bit register, shifted by w positions: site m is stored at position
// p = m + w.  At iteration t every lane therefore needs position t, i.e.
// register t / 6, field t % 6 -- a static index in the fully unrolled loop.
//
// Couplings: one producer warp streams the row of the step's site through a
// ring of 4 chunk slots of 32 sites, each slot [q*q cells][32 sites] floats
// (cell row a*q + b: 128 bytes, all 32 banks), filled by one 1-D bulk copy
// per chunk.  (Ring layouts interleaved per cell need one copy per cell row:
// 128-byte bulk copies or 16-byte cp.async then feed a slot at <= 30 GB/s
// per SM, while chunk-sized bulk copies reach > 200 GB/s per SM.)  The global layout (mi3_unpack_j_tiles) holds, for each site pos,
// NC = ceil((L + 31) / 32) chunks of [q*q cells][32 sites], zero on the
// diagonal (m == pos, the reference's skipped site) and for sites >= L.  A
// lane that runs ahead past site L - 1 (end of a step) or lags behind site 0
// (start of a step, reading the previous step's last chunk) finds zero
// couplings and zero residues there: it adds exact zeros, so no lane needs a
// mask.  Adding +0 leaves a float sum unchanged, as the zero diagonal does.
#include <algorithm>

#include "common.cuh"

namespace mi3 {

constexpr uint32_t SKEW_SLOTS = 4;
constexpr uint32_t SKEW_HEAD = 128;              // mbarriers + abort flag

inline uint32_t skew_chunks(uint32_t L) { return (L + 31 + 31) / 32; }

// T[pos][k][a*q + b][c] = J_{pos,m}(a, b), m = 32 k + c (0 for m == pos or m >= L).
__global__ void k_unpack_j_tiles(const float *__restrict__ J, float *__restrict__ T, uint32_t L, uint32_t q,
                                 uint32_t nc) {
    const uint32_t pos = blockIdx.y, qq = q * q;
    const uint64_t row_len = (uint64_t)nc * qq * 32;
    float *row = T + (uint64_t)pos * row_len;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < row_len;
         k += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t chunk = (uint32_t)(k / (qq * 32));
        const uint32_t r = (uint32_t)(k - (uint64_t)chunk * qq * 32);
        const uint32_t cell = r >> 5, m = chunk * 32 + (r & 31);
        const uint32_t a = cell / q, b = cell - a * q;
        float v = 0.0f;
        if (m < L && m != pos) {
            if (pos < m) {
                const uint64_t n = (uint64_t)pos * (2 * L - pos - 1) / 2 + (m - pos - 1);
                v = J[n * qq + a * q + b];
            } else {
                const uint64_t n = (uint64_t)m * (2 * L - m - 1) / 2 + (pos - m - 1);
                v = J[n * qq + b * q + a];
            }
        }
        row[k] = v;
    }
}

struct SkewParams {
    const float *Jt;
    uint64_t row_floats;  // floats per site row of Jt
    uint64_t replica_floats;  // floats between replicas of the table (0: one table)
    uint32_t replicas;
    uint4 *rng;
    const uint32_t *poslist;
    uint32_t pos_off;
    uint32_t nsteps;
    const float *betas;
    float beta;
    uint32_t *seq;
    uint32_t nseqs;
    uint32_t L, q;
    uint32_t nc;  // chunks per row
    int32_t *status;
};

// k == idx ? a : b, kept as a per-register select (written as PTX so that
// the compiler does not fold a chain of them into an indexed access, which
// would move the register array to local memory).
__device__ __forceinline__ uint32_t sel_eq(uint32_t idx, uint32_t k, uint32_t a, uint32_t b) {
    uint32_t r;
    asm("{\n\t.reg .pred p;\n\tsetp.eq.u32 p, %1, %2;\n\tselp.b32 %0, %3, %4, p;\n\t}"
        : "=r"(r)
        : "r"(idx), "r"(k), "r"(a), "r"(b));
    return r;
}

// (residue at field F of word w) * 128: the byte offset of its cell row
// (rows of 32 floats) relative to the row of residue 0.
template <uint32_t F>
__device__ __forceinline__ uint32_t res_row_bytes(uint32_t w) {
    constexpr int SH = 7 - 5 * (int)F;
    if constexpr (SH >= 0)
        return (w << SH) & (31u << 7);
    else
        return (w >> (-SH)) & (31u << 7);
}

template <uint32_t OFF>
__device__ __forceinline__ float lds_f32_off(uint32_t addr) {
    float v;
    asm volatile("ld.shared.f32 %0, [%1+%2];" : "=f"(v) : "r"(addr), "n"(OFF));
    return v;
}

// Per-body addressing.  Lane w at iteration t = 32 B + tau reads site
// t - w: for tau >= w that is column tau - w of chunk G (this body's
// chunk, slot base pc), otherwise column tau - w + 32 of chunk G - 1
// (slot base pp).  qc = pc - 4 w and qp = pp + 128 - 4 w, so the column's
// byte address is (tau >= w ? qc : qp) + 4 tau, the 4 tau going into the
// load's immediate offset.
struct SkewBody {
    uint32_t qc, qp, baseA, baseB, lane;
};

// One loop iteration (static TAU within body B; T = 32 B + TAU): add the
// lane's site term to dE.
template <uint32_t NW, uint32_t T>
__device__ __forceinline__ void skew_term(const uint32_t (&sq)[NW], const SkewBody &bd, float &dE) {
    if constexpr (T < 6 * NW) {
        constexpr uint32_t TAU = T % 32;
        const uint32_t q = (TAU >= bd.lane) ? bd.qc : bd.qp;
        const uint32_t x = res_row_bytes<T % 6>(sq[T / 6]) + q;
        const float a = lds_f32_off<4 * TAU>(bd.baseA + x);
        const float b = lds_f32_off<4 * TAU>(bd.baseB + x);
        dE += a - b;
    }
}

// Eight iterations starting at T0.
template <uint32_t NW, uint32_t T0>
__device__ __forceinline__ void skew_eight(const uint32_t (&sq)[NW], const SkewBody &bd, float &dE) {
    skew_term<NW, T0 + 0>(sq, bd, dE);
    skew_term<NW, T0 + 1>(sq, bd, dE);
    skew_term<NW, T0 + 2>(sq, bd, dE);
    skew_term<NW, T0 + 3>(sq, bd, dE);
    skew_term<NW, T0 + 4>(sq, bd, dE);
    skew_term<NW, T0 + 5>(sq, bd, dE);
    skew_term<NW, T0 + 6>(sq, bd, dE);
    skew_term<NW, T0 + 7>(sq, bd, dE);
}

// Body B: iterations 32 B .. 32 B + 31 (those below tend), which read
// chunks G - 1 and G.
template <uint32_t NW, uint32_t B>
__device__ __forceinline__ void skew_body(const uint32_t (&sq)[NW], const SkewBody &bd, uint32_t tend, float &dE) {
    skew_eight<NW, 32 * B + 0>(sq, bd, dE);
    if (32 * B + 8 >= tend) return;
    skew_eight<NW, 32 * B + 8>(sq, bd, dE);
    if (32 * B + 16 >= tend) return;
    skew_eight<NW, 32 * B + 16>(sq, bd, dE);
    if (32 * B + 24 >= tend) return;
    skew_eight<NW, 32 * B + 24>(sq, bd, dE);
}

struct SkewStep {
    uint64_t *full, *empty;
    volatile int *abort_flag;
    int32_t *status;
    uint32_t G0, lane, tend;
    uint32_t ring_s, slot_bytes;
};

// Wait for chunk G, run body B, release chunk G - 1.  Returns false when a
// bounded wait gave up.
template <uint32_t NW, uint32_t B>
__device__ __forceinline__ bool skew_run_body(const SkewStep &st, const uint32_t (&sq)[NW], uint32_t baseA,
                                              uint32_t baseB, float &dE) {
    const uint32_t G = st.G0 + B;
    // every lane waits (each acquires the bulk-copied data); the verdict is
    // made warp-uniform so that no lane is left behind at __syncwarp
    const bool w = mbar_wait_bounded(&st.full[G & 3], ((G - 1) >> 2) & 1, st.abort_flag, WAIT_LIMIT_NS);
    if (!__all_sync(0xffffffffu, w)) {
        if (st.lane == 0) {
            if (!*st.abort_flag) report(st.status, ST_TIMEOUT_FULL);
            *st.abort_flag = 1;
        }
        return false;
    }
    SkewBody bd;
    bd.qc = st.ring_s + (G & 3) * st.slot_bytes - 4 * st.lane;
    bd.qp = st.ring_s + ((G - 1) & 3) * st.slot_bytes + 128 - 4 * st.lane;
    bd.baseA = baseA;
    bd.baseB = baseB;
    bd.lane = st.lane;
    skew_body<NW, B>(sq, bd, st.tend, dE);
    __syncwarp();
    if (st.lane == 0) mbar_arrive(&st.empty[(G - 1) & 3]);
    return true;
}

template <uint32_t NW, uint32_t B>
__device__ __forceinline__ bool skew_bodies(const SkewStep &st, const uint32_t (&sq)[NW], uint32_t baseA,
                                            uint32_t baseB, float &dE) {
    if constexpr (32 * B < 6 * NW) {
        if (32 * B >= st.tend) return true;
        if (!skew_run_body<NW, B>(st, sq, baseA, baseB, dE)) return false;
        return skew_bodies<NW, B + 1>(st, sq, baseA, baseB, dE);
    } else {
        return true;
    }
}

// NW: sequence registers per lane (6 * NW >= L + 31); WARPS: consumer warps.
// Register cap: each of the SM's 4 schedulers owns a quarter of the register
// file (16384 registers) and holds every fourth warp, so with WARPS + 1 = 17
// warps one scheduler holds 5 (5 x 32 x 96 <= 16384), with 25 warps 7
// (7 x 32 x 72 <= 16384) and with 9 warps 3 (3 x 32 x 168 <= 16384) -- the
// 8-warp kernel has room for the 91 sequence registers of L = 512.
template <uint32_t NW, uint32_t WARPS>
__global__ void __maxnreg__(WARPS == 8 ? 168 : (WARPS == 16 ? 96 : 72)) k_metropolis_skew(const SkewParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *full = reinterpret_cast<uint64_t *>(smem);
    uint64_t *empty = full + SKEW_SLOTS;
    volatile int *abort_flag = reinterpret_cast<volatile int *>(empty + SKEW_SLOTS);
    float *ring = reinterpret_cast<float *>(smem + SKEW_HEAD);
    uint32_t *stage = reinterpret_cast<uint32_t *>(ring);  // sequence staging, before and after the loop

    constexpr uint32_t NWALK = 32 * WARPS;
    constexpr uint32_t STR = NW + 1;  // staging words per walker (odd: few bank conflicts)
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t qq = p.q * p.q;
    const uint32_t slot_bytes = qq * 128;            // one chunk: [q*q cells][32 sites] floats
    const uint32_t g = blockIdx.x * NWALK + tid;  // this consumer's walker
    // the last CTA may be partly filled: lanes past nseqs run on a zero
    // sequence and store nothing
    const bool valid = g < p.nseqs;

    if (tid == 0) {
        for (uint32_t s = 0; s < SKEW_SLOTS; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], WARPS);
        }
        *abort_flag = 0;
        fence_mbar_init();
    }

    // ---- the walkers' sequences -> lane-shifted 5-bit registers
    uint32_t sq[NW];
#pragma unroll
    for (uint32_t k = 0; k < NW; ++k) sq[k] = 0;
    if (warp < WARPS) {
        uint32_t *my = stage + tid * STR;
        for (uint32_t k = 0; k < NW; ++k) my[k] = 0;
        uint32_t gw = 0;
        for (uint32_t m = 0; m < p.L && valid; ++m) {
            if ((m & 3) == 0) gw = p.seq[(size_t)(m >> 2) * p.nseqs + g];
            // residues >= q (invalid input) are clamped to q - 1 so every
            // cell row stays inside the ring
            const uint32_t r = min(getbyte(gw, m & 3), p.q - 1);
            const uint32_t pp = m + lane;
            my[pp / 6] |= r << (5 * (pp % 6));
        }
#pragma unroll
        for (uint32_t k = 0; k < NW; ++k) sq[k] = my[k];
    }
    __syncthreads();
    // slot 0 starts as a chunk of zeros: the first step's lagging lanes read it
    for (uint32_t c = tid; c < qq * 32; c += blockDim.x) ring[c] = 0.0f;
    fence_proxy_async_smem();
    __syncthreads();

    const uint32_t ring_s = smem_addr(ring);
    if (warp == WARPS) {
        // ---------------------------------------------------- producer warp
        uint32_t G = 1;  // global chunk index; chunk 0 is the zero slot
        bool ok = true;
        for (uint32_t i = 0; i < p.nsteps && ok; ++i) {
            uint32_t pos = __ldg(&p.poslist[p.pos_off + i]);
            if (pos >= p.L) pos = 0;  // invalid site: consumers report it
            const float *row = p.Jt + (uint64_t)(blockIdx.x % p.replicas) * p.replica_floats +
                               (uint64_t)pos * p.row_floats;
            for (uint32_t k = 0; k < p.nc; ++k, ++G) {
                const uint32_t s = G & 3;
                if (G >= SKEW_SLOTS) {
                    int w = 1;
                    if (lane == 0) {
                        w = mbar_wait_bounded(&empty[s], ((G - SKEW_SLOTS) >> 2) & 1, abort_flag, WAIT_LIMIT_NS);
                        if (!w) {
                            if (!*abort_flag) report(p.status, ST_TIMEOUT_EMPTY);
                            *abort_flag = 1;
                        }
                    }
                    if (!__shfl_sync(0xffffffffu, w, 0)) {
                        ok = false;
                        break;
                    }
                }
                // one bulk copy per chunk: the chunk is contiguous in global
                // memory and fills its slot as it is
                if (lane == 0) {
                    mbar_arrive_expect_tx(&full[s], slot_bytes);
                    bulk_g2s(ring + (size_t)s * (slot_bytes / 4), row + (uint64_t)k * qq * 32, slot_bytes, &full[s]);
                }
                __syncwarp();
            }
        }
        // Drain: every copy issued must land before the CTA may reuse the
        // ring.
        if (lane == 0) {
            const uint32_t first = G > SKEW_SLOTS + 1 ? G - SKEW_SLOTS : 1;
            for (uint32_t gg = first; gg < G; ++gg)
                mbar_wait_bounded(&full[gg & 3], ((gg - 1) >> 2) & 1, nullptr, WAIT_LIMIT_NS);
        }
        __syncwarp();
    } else {
        // -------------------------------------------------------- consumers
        uint4 s4 = valid ? p.rng[g] : make_uint4(1, 1, 1, 1);
        Rng2 rng{s4.x, s4.y, s4.z, s4.w};
        const float Bta = (p.betas && valid) ? p.betas[g] : p.beta;
        SkewStep st{full, empty, abort_flag, p.status, 1, lane, p.L + 31, ring_s, slot_bytes};
        for (uint32_t i = 0; i < p.nsteps; ++i, st.G0 += p.nc) {
            uint32_t pos = __ldg(&p.poslist[p.pos_off + i]);
            if (pos >= p.L) {
                report(p.status, ST_BAD_INPUT);
                pos = 0;
            }
            uint32_t r0, r1;
            rng_next2(rng, r0, r1);
            const uint32_t mut = r0 % p.q;
            const uint32_t pp = pos + lane, wi = pp / 6, sh = 5 * (pp - 6 * wi);
            uint32_t word = 0;
#pragma unroll
            for (uint32_t k = 0; k < NW; ++k) word = sel_eq(wi, k, sq[k], word);
            const uint32_t cur = (word >> sh) & 31u;
            // byte offsets of the cell rows (a = mut or cur, b = 0) in a slot
            const uint32_t baseA = mut * p.q * 128, baseB = cur * p.q * 128;
            float dE = 0.0f;
            if (!skew_bodies<NW, 0>(st, sq, baseA, baseB, dE)) break;
            const float x = -Bta * dE;
            const bool acc = accept_exp(x, uniform_map(r1));
            const uint32_t nw = acc ? ((word & ~(31u << sh)) | (mut << sh)) : word;
#pragma unroll
            for (uint32_t k = 0; k < NW; ++k) sq[k] = sel_eq(wi, k, nw, sq[k]);
        }
        if (valid) p.rng[g] = make_uint4(rng.x0, rng.x1, rng.c0, rng.c1);
    }

    // ---- registers -> sequences (the ring is idle: every copy has landed)
    __syncthreads();
    if (warp < WARPS && valid) {
        uint32_t *my = stage + tid * STR;
#pragma unroll
        for (uint32_t k = 0; k < NW; ++k) my[k] = sq[k];
        uint32_t gw = 0;
        for (uint32_t m = 0; m < p.L; ++m) {
            const uint32_t pp = m + lane;
            gw = setbyte(gw, m & 3, (my[pp / 6] >> (5 * (pp % 6))) & 31u);
            if ((m & 3) == 3 || m == p.L - 1) {
                p.seq[(size_t)(m >> 2) * p.nseqs + g] = gw;
                gw = 0;
            }
        }
    }
}

using SkewKernel = void (*)(const SkewParams);

template <uint32_t WARPS>
static SkewKernel skew_kernel_for(uint32_t nw) {
    switch (nw) {
        case 8: return k_metropolis_skew<8, WARPS>;
        case 16: return k_metropolis_skew<16, WARPS>;
        case 24: return k_metropolis_skew<24, WARPS>;
        case 32: return k_metropolis_skew<32, WARPS>;
        case 40: return k_metropolis_skew<40, WARPS>;
        case 44: return k_metropolis_skew<44, WARPS>;
        case 48: return k_metropolis_skew<48, WARPS>;
        default: return nullptr;
    }
}

// Longer sequences: the 8-warp kernel only.
static SkewKernel skew_kernel_long(uint32_t nw) {
    switch (nw) {
        case 56: return k_metropolis_skew<56, 8>;
        case 64: return k_metropolis_skew<64, 8>;
        case 72: return k_metropolis_skew<72, 8>;
        case 80: return k_metropolis_skew<80, 8>;
        case 88: return k_metropolis_skew<88, 8>;
        case 96: return k_metropolis_skew<96, 8>;
        default: return skew_kernel_for<8>(nw);
    }
}

// Sequence registers for L: the smallest instantiated NW with 6 NW >= L + 31
// (at most 48 with 512 or 768 walkers per CTA, 96 with 256).
static uint32_t skew_nw(uint32_t L, uint32_t max_nw) {
    const uint32_t nws[13] = {8, 16, 24, 32, 40, 44, 48, 56, 64, 72, 80, 88, 96};
    for (uint32_t nw : nws)
        if (nw <= max_nw && 6 * nw >= L + 31) return nw;
    return 0;
}

static size_t skew_smem(uint32_t q, uint32_t nw, uint32_t warps) {
    const size_t ring = (size_t)SKEW_SLOTS * q * q * 128;
    const size_t staging = (size_t)32 * warps * (nw + 1) * 4;
    return SKEW_HEAD + std::max(ring, staging);
}

}  // namespace mi3

using namespace mi3;

extern "C" uint64_t mi3_jtiles_floats(uint32_t L, uint32_t q) {
    if (L < 2 || q < 1) return 0;
    return (uint64_t)L * skew_chunks(L) * q * q * 32;
}

extern "C" int mi3_unpack_j_tiles(const float *J, float *Jtiles, uint32_t L, uint32_t q, void *stream) {
    if (!J || !Jtiles) return fail(MI3_ERR_ARG, "mi3_unpack_j_tiles: null pointer");
    if (L < 2 || q < 1 || q > 255) return fail(MI3_ERR_ARG, "mi3_unpack_j_tiles: bad L/q");
    if (!aligned(Jtiles, 16)) return fail(MI3_ERR_ALIGN, "mi3_unpack_j_tiles: Jtiles not 16B aligned");
    const uint32_t nc = skew_chunks(L);
    const uint64_t row = (uint64_t)nc * q * q * 32;
    const uint32_t tb = 256;
    const uint32_t gx = (uint32_t)std::min<uint64_t>((row + tb - 1) / tb, 1024);
    k_unpack_j_tiles<<<dim3(gx, L), tb, 0, as_stream(stream)>>>(J, Jtiles, L, q, nc);
    return check_launch("mi3_unpack_j_tiles");
}

extern "C" int mi3_metropolis_skew(const float *Jtiles, uint32_t *rngstates, uint32_t position_offset,
                                   const uint32_t *position_list, uint32_t nsteps, const float *betas, float beta,
                                   uint32_t *seqmem, uint32_t nseqs, uint32_t L, uint32_t q,
                                   uint32_t walkers_per_cta, uint32_t replicas, int32_t *status, void *stream) {
    if (!Jtiles || !rngstates || !position_list || !seqmem || !status)
        return fail(MI3_ERR_ARG, "mi3_metropolis_skew: null pointer");
    if (L < 2 || q < 2 || q > 21) return fail(MI3_ERR_ARG, "mi3_metropolis_skew: needs 2 <= q <= 21");
    if (walkers_per_cta == 0) walkers_per_cta = L + 31 <= 6 * 48 ? 512 : 256;
    if (walkers_per_cta != 256 && walkers_per_cta != 512 && walkers_per_cta != 768)
        return fail(MI3_ERR_ARG, "mi3_metropolis_skew: walkers per CTA must be 256, 512 or 768");
    const uint32_t nw = skew_nw(L, walkers_per_cta == 256 ? 96 : 48);
    if (!nw)
        return fail(MI3_ERR_ARG, "mi3_metropolis_skew: L too large (L + 31 <= 288, or <= 576 with 256 walkers per CTA)");
    if (nseqs == 0 || nseqs % 32)
        return fail(MI3_ERR_ARG, "mi3_metropolis_skew: nseqs must be a positive multiple of 32");
    if (!aligned(Jtiles, 16) || !aligned(rngstates, 16))
        return fail(MI3_ERR_ALIGN, "mi3_metropolis_skew: Jtiles/rngstates must be 16B aligned");
    if (nsteps == 0) return MI3_OK;
    const uint32_t warps = walkers_per_cta / 32;
    SkewKernel kernel = warps == 8 ? skew_kernel_long(nw) : warps == 16 ? skew_kernel_for<16>(nw) : skew_kernel_for<24>(nw);
    const size_t smem = skew_smem(q, nw, warps);
    if (!kernel || smem > 227 * 1024) return fail(MI3_ERR_ARG, "mi3_metropolis_skew: shape exceeds the kernel's limits");
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    SkewParams p;
    p.Jt = Jtiles;
    p.row_floats = (uint64_t)skew_chunks(L) * q * q * 32;
    p.replicas = replicas ? replicas : 1;
    p.replica_floats = mi3_jtiles_floats(L, q);
    p.rng = reinterpret_cast<uint4 *>(rngstates);
    p.poslist = position_list;
    p.pos_off = position_offset;
    p.nsteps = nsteps;
    p.betas = betas;
    p.beta = beta;
    p.seq = seqmem;
    p.nseqs = nseqs;
    p.L = L;
    p.q = q;
    p.nc = skew_chunks(L);
    p.status = status;
    kernel<<<(nseqs + walkers_per_cta - 1) / walkers_per_cta, walkers_per_cta + 32, smem, as_stream(stream)>>>(p);
    return check_launch("mi3_metropolis_skew");
}
