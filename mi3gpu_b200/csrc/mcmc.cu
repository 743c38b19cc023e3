// mcmc.cu -- coupling unpacking and the Metropolis sampler.
//
// Sampler design (B200): one walker per consumer thread, NW walkers per CTA.
// Each walker's packed sequence lives in shared memory for the whole launch
// (loaded once, stored once), so HBM sees the sequences twice per launch
// instead of once per step.  All walkers of the launch share the site
// sequence (position_list), so every CTA needs the same coupling row
// Jrows[pos] (L blocks of q*q floats) at every step.  One producer warp
// streams that row through an S-stage shared-memory ring with 1-D bulk
// copies (cp.async.bulk, completion on mbarriers); the row stays hot in L2
// (the whole unpacked table is < L2 at L=232, q=21).  Consumers gather the
// two entries J[pos][m][mut][s_m] and J[pos][m][cur][s_m] per site m from the
// staged chunk and accumulate dE in site order, as DeltaEnergy does
// (mcmc.cl:360-413).
#include <algorithm>

#include "common.cuh"

namespace mi3 {

// ----------------------------------------------------------------- unpack J
// Jrows[i][j][a][b] = J_ij(a,b) for i<j, J_ji(b,a) for i>j, 0 on the diagonal
// and in the row padding (unpackfV, mcmc.cl:42-65).
__global__ void k_unpack_j(const float *__restrict__ J, float *__restrict__ Jrows, uint32_t L,
                           uint32_t q, uint64_t stride) {
    uint32_t i = blockIdx.y;
    uint32_t qq = q * q;
    const uint64_t row_len = stride;
    float *row = Jrows + (uint64_t)i * stride;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < row_len;
         k += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t j = (uint32_t)(k / qq);
        uint32_t li = (uint32_t)(k - (uint64_t)j * qq);
        float v = 0.0f;
        if (j < L && j != i) {
            if (i < j) {
                uint64_t n = (uint64_t)i * (2 * L - i - 1) / 2 + (j - i - 1);
                v = J[n * qq + li];
            } else {
                uint64_t n = (uint64_t)j * (2 * L - j - 1) / 2 + (i - j - 1);
                v = J[n * qq + q * (li % q) + li / q];
            }
        }
        row[k] = v;
    }
}

// ---------------------------------------------------------------- sampler
struct MetroParams {
    const float *Jrows;
    uint64_t stride;  // floats per row
    uint4 *rng;
    const uint32_t *poslist;
    uint32_t pos_off;
    uint32_t nsteps;
    const float *betas;
    float beta;
    uint32_t *seq;
    uint32_t nseqs;
    uint32_t L, q;
    uint32_t M;        // sites per chunk (multiple of 4)
    uint32_t nchunks;  // ceil(L / M)
    uint32_t stages;
    uint32_t stage_floats;  // floats per stage buffer (multiple of 32)
    int32_t *status;
};

// Shared memory: [full mbarriers S][empty mbarriers S][abort flag] (pad 128)
//                [stage buffers S * stage_floats][pad STAGE_PAD][seq words ceil(L/PK) * NW]
// The pad absorbs gathers with an out-of-range residue byte (< 256 floats).
//
// PK residues per shared-memory word: 4 (bytes, the global layout) or, for
// q <= 32, 6 (5 bits each) -- a walker's sequence then takes 2/3 of the
// space, so more walkers fit per SM and a site block costs fewer word
// loads.  The packing is internal: the kernel converts from and to the
// global byte layout when it loads and stores the walkers, and the float
// sums run over the same sites in the same order.
constexpr uint32_t STAGE_PAD = 256;

template <uint32_t PK>
__device__ __forceinline__ uint32_t res_get(uint32_t w, uint32_t k) {
    constexpr uint32_t BITS = PK == 4 ? 8 : 5;
    return (w >> (BITS * k)) & ((1u << BITS) - 1);
}

template <uint32_t PK>
__device__ __forceinline__ uint32_t res_set(uint32_t w, uint32_t k, uint32_t v) {
    constexpr uint32_t BITS = PK == 4 ? 8 : 5, MASK = (1u << BITS) - 1;
    return (w & ~(MASK << (BITS * k))) | ((v & MASK) << (BITS * k));
}

template <uint32_t PK>
__global__ void __launch_bounds__(544, 1) k_metropolis(const MetroParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    const uint32_t NW = blockDim.x - 32;  // consumer threads = walkers
    const uint32_t S = p.stages;
    uint64_t *full = reinterpret_cast<uint64_t *>(smem);
    uint64_t *empty = full + S;
    volatile int *abort_flag = reinterpret_cast<volatile int *>(empty + S);
    float *stage = reinterpret_cast<float *>(smem + 128 * ((16 * S + 4 + 127) / 128));
    uint32_t *seq_s = reinterpret_cast<uint32_t *>(stage + (size_t)S * p.stage_floats + STAGE_PAD);

    const uint32_t tid = threadIdx.x;
    const uint32_t warp = tid >> 5, lane = tid & 31;
    const uint32_t qq = p.q * p.q;
    const uint32_t sw = (p.L - 1) / 4 + 1;  // global words (4 residues each)

    if (tid == 0) {
        for (uint32_t s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], NW / 32);
        }
        *abort_flag = 0;
        fence_mbar_init();
    }
    __syncthreads();

    if (warp == NW / 32) {
        // ---------------------------------------------------- producer warp
        if (lane == 0) {
            uint32_t k = 0;
            bool ok = true;
            for (uint32_t i = 0; i < p.nsteps && ok; ++i) {
                uint32_t pos = __ldg(&p.poslist[p.pos_off + i]);
                if (pos >= p.L) pos = 0;  // invalid site: consumers report it
                const float *row = p.Jrows + (uint64_t)pos * p.stride;
                for (uint32_t c = 0; c < p.nchunks; ++c, ++k) {
                    uint32_t s = k % S;
                    if (k >= S) {
                        uint32_t ph = ((k / S) - 1) & 1;
                        if (!mbar_wait_bounded(&empty[s], ph, abort_flag, WAIT_LIMIT_NS)) {
                            if (!*abort_flag) report(p.status, ST_TIMEOUT_EMPTY);
                            *abort_flag = 1;
                            ok = false;
                            break;
                        }
                    }
                    uint32_t m0 = c * p.M;
                    uint32_t nm = min(p.M, p.L - m0);
                    uint32_t bytes = (nm * qq * 4 + 15) & ~15u;
                    mbar_arrive_expect_tx(&full[s], bytes);
                    bulk_g2s(stage + (size_t)s * p.stage_floats, row + (uint64_t)m0 * qq, bytes,
                             &full[s]);
                }
            }
            // Drain: every copy issued must land before the CTA may exit.
            uint32_t first = k > S ? k - S : 0;
            for (uint32_t kk = first; kk < k; ++kk)
                mbar_wait_bounded(&full[kk % S], (kk / S) & 1, nullptr, WAIT_LIMIT_NS);
        }
        return;
    }

    // -------------------------------------------------------- consumers
    const uint32_t g = blockIdx.x * NW + tid;
    if constexpr (PK == 4) {
        for (uint32_t w = 0; w < sw; ++w) seq_s[w * NW + tid] = p.seq[(size_t)w * p.nseqs + g];
    } else {
        uint32_t gw = 0, acc = 0;
        for (uint32_t j = 0; j < p.L; ++j) {
            if ((j & 3) == 0) gw = p.seq[(size_t)(j >> 2) * p.nseqs + g];
            const uint32_t k = j % PK;
            acc = res_set<PK>(acc, k, getbyte(gw, j & 3));
            if (k == PK - 1 || j == p.L - 1) {
                seq_s[(j / PK) * NW + tid] = acc;
                acc = 0;
            }
        }
    }
    uint4 s4 = p.rng[g];
    Rng2 rng{s4.x, s4.y, s4.z, s4.w};
    const float B = p.betas ? p.betas[g] : p.beta;
    // seq_s is private per thread (column tid), no barrier needed.

    uint32_t k = 0;
    bool ok = true;
    for (uint32_t i = 0; i < p.nsteps && ok; ++i) {
        uint32_t pos = __ldg(&p.poslist[p.pos_off + i]);
        if (pos >= p.L) {
            report(p.status, ST_BAD_INPUT);
            pos = 0;
        }
        uint32_t r0, r1;
        rng_next2(rng, r0, r1);
        uint32_t mut = r0 % p.q;
        const uint32_t pw = pos / PK, pk = pos - pw * PK;
        uint32_t wpos = seq_s[pw * NW + tid];
        // residues are < q for valid input; the clamp keeps an invalid one
        // inside the stage buffer (an out-of-range s_m lands in the pad).
        uint32_t cur = min(res_get<PK>(wpos, pk), p.q - 1);
        uint32_t mq = mut * p.q, cq = cur * p.q;
        float dE = 0.0f;
        for (uint32_t c = 0; c < p.nchunks; ++c, ++k) {
            uint32_t s = k % S;
            if (!mbar_wait_bounded(&full[s], (k / S) & 1, abort_flag, WAIT_LIMIT_NS)) {
                if (!*abort_flag) report(p.status, ST_TIMEOUT_FULL);
                *abort_flag = 1;
                ok = false;
                break;
            }
            const float *Jc = stage + (size_t)s * p.stage_floats;
            uint32_t m0 = c * p.M;  // a multiple of PK
            uint32_t nm = min(p.M, p.L - m0);
            uint32_t nfull = nm / PK;
            const uint32_t *sq = seq_s + (m0 / PK) * NW + tid;
#pragma unroll 2
            for (uint32_t w = 0; w < nfull; ++w) {
                uint32_t word = sq[w * NW];
                const float *Jm = Jc + w * PK * qq;
#pragma unroll
                for (uint32_t b = 0; b < PK; ++b) {
                    uint32_t sm = res_get<PK>(word, b);
                    dE += Jm[b * qq + mq + sm] - Jm[b * qq + cq + sm];
                }
            }
            uint32_t rem = nm - nfull * PK;
            if (rem) {
                uint32_t word = sq[nfull * NW];
                const float *Jm = Jc + nfull * PK * qq;
                for (uint32_t b = 0; b < rem; ++b) {
                    uint32_t sm = res_get<PK>(word, b);
                    dE += Jm[b * qq + mq + sm] - Jm[b * qq + cq + sm];
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[s]);
        }
        if (!ok) break;
        float x = -B * dE;
        if (accept_exp(x, uniform_map(r1))) seq_s[pw * NW + tid] = res_set<PK>(wpos, pk, mut);
    }
    if constexpr (PK == 4) {
        for (uint32_t w = 0; w < sw; ++w) p.seq[(size_t)w * p.nseqs + g] = seq_s[w * NW + tid];
    } else {
        uint32_t gw = 0, sword = 0;
        for (uint32_t j = 0; j < p.L; ++j) {
            const uint32_t k = j % PK;
            if (k == 0) sword = seq_s[(j / PK) * NW + tid];
            gw = setbyte(gw, j & 3, res_get<PK>(sword, k));
            if ((j & 3) == 3 || j == p.L - 1) {
                p.seq[(size_t)(j >> 2) * p.nseqs + g] = gw;
                gw = 0;
            }
        }
    }
    p.rng[g] = make_uint4(rng.x0, rng.x1, rng.c0, rng.c1);
}

struct MetroConfig {
    uint32_t NW, M, nchunks, stages, stage_floats;
    size_t smem;
    uint32_t pk;  // residues per shared-memory word
};

// 5-bit residues when they fit and chunks start on whole words of 6
static uint32_t metro_pk(uint32_t q, uint32_t M) { return (q <= 32 && M % 12 == 0) ? 6 : 4; }

static size_t metro_smem(uint32_t NW, uint32_t S, uint32_t stage_floats, uint32_t L, uint32_t pk) {
    size_t head = 128 * ((16 * S + 4 + 127) / 128);
    return head + (size_t)S * stage_floats * 4 + STAGE_PAD * 4 + (size_t)((L + pk - 1) / pk) * NW * 4;
}

// Sites per chunk for a stage of about `bytes`: a multiple of 4 (16-byte
// aligned bulk copies), of 12 when q <= 32 (whole 5-bit words), at most the
// rounded row.
static uint32_t metro_chunk(uint32_t L, uint32_t q, uint32_t bytes) {
    const uint32_t Lr = (L + 3) & ~3u;
    uint32_t M = bytes / (q * q * 4);
    const uint32_t unit = (q <= 32 && M >= 12) ? 12 : 4;
    M = std::max<uint32_t>(4, M - M % unit);
    return std::min(M, Lr);
}

static bool pick_metro_config(uint32_t L, uint32_t q, uint32_t nseqs, MetroConfig &cfg) {
    const size_t SMEM_MAX = 227 * 1024;
    const uint32_t qq = q * q;
    // sites per chunk: stages of up to ~48 KB, at most the (rounded) row;
    // two stages first.  (Timing every plan at L=232/512, q=21 put two or
    // three ~40 KB stages first: fewer, larger bulk copies per coupling row
    // beat a deeper ring of small ones.)
    const uint32_t M = metro_chunk(L, q, 48 * 1024);
    const uint32_t step = metro_pk(q, M) == 6 ? 12 : 4;
    uint32_t cands[4] = {512, 384, 256, 128};
    for (uint32_t NW : cands) {
        if (nseqs % NW) continue;
        // prefer enough CTAs to fill the SMs when walkers are few
        if (NW > 128 && nseqs / NW < 148) continue;
        for (uint32_t S = 2; S <= 4; ++S) {
            for (uint32_t m = M; m >= step; m -= step) {
                uint32_t stage_floats = ((m * qq) + 31) & ~31u;
                const uint32_t pk = metro_pk(q, m);
                size_t sm = metro_smem(NW, S, stage_floats, L, pk);
                if (sm <= SMEM_MAX) {
                    cfg = MetroConfig{NW, m, (L + m - 1) / m, S, stage_floats, sm, pk};
                    return true;
                }
            }
        }
    }
    return false;
}

}  // namespace mi3

using namespace mi3;

extern "C" int mi3_unpack_j(const float *J, float *Jrows, uint32_t L, uint32_t q, void *stream) {
    if (!J || !Jrows) return fail(MI3_ERR_ARG, "mi3_unpack_j: null pointer");
    if (L < 2 || q < 1 || q > 255) return fail(MI3_ERR_ARG, "mi3_unpack_j: bad L/q");
    if (!aligned(Jrows, 16)) return fail(MI3_ERR_ALIGN, "mi3_unpack_j: Jrows not 16B aligned");
    uint64_t stride = jrow_stride(L, q);
    uint32_t tb = 256;
    uint32_t gx = (uint32_t)std::min<uint64_t>((stride + tb - 1) / tb, 1024);
    dim3 grid(gx, L);
    k_unpack_j<<<grid, tb, 0, as_stream(stream)>>>(J, Jrows, L, q, stride);
    return check_launch("mi3_unpack_j");
}

namespace mi3 {

// A caller-chosen plan (walkers per CTA, sites per chunk, stages), checked
// against the kernel's limits; zeros leave the choice to pick_metro_config.
static int make_metro_config(uint32_t L, uint32_t q, uint32_t nseqs, uint32_t NW, uint32_t M, uint32_t S,
                             MetroConfig &cfg) {
    if (NW == 0 && M == 0 && S == 0) {
        if (!pick_metro_config(L, q, nseqs, cfg))
            return fail(MI3_ERR_ARG, "mi3_metropolis: L/q too large for the shared-memory plan");
        return MI3_OK;
    }
    const uint32_t Lr = (L + 3) & ~3u, qq = q * q;
    if (NW < 64 || NW > 512 || NW % 32 || nseqs % NW)
        return fail(MI3_ERR_ARG, "mi3_metropolis: walkers per CTA must be a multiple of 32 in [64, 512] dividing nseqs");
    if (M < 4 || M % 4 || M > Lr) return fail(MI3_ERR_ARG, "mi3_metropolis: sites per chunk must be a multiple of 4 <= L");
    if (S < 2 || S > 8) return fail(MI3_ERR_ARG, "mi3_metropolis: stages must be in [2, 8]");
    const uint32_t stage_floats = ((M * qq) + 31) & ~31u;
    const uint32_t pk = metro_pk(q, M);
    const size_t sm = metro_smem(NW, S, stage_floats, L, pk);
    if (sm > 227 * 1024) return fail(MI3_ERR_ARG, "mi3_metropolis: plan exceeds shared memory");
    cfg = MetroConfig{NW, M, (L + M - 1) / M, S, stage_floats, sm, pk};
    return MI3_OK;
}

}  // namespace mi3

extern "C" uint32_t mi3_metropolis_plans(uint32_t L, uint32_t q, uint32_t nseqs, uint32_t *plans, uint32_t max) {
    uint32_t n = 0;
    if (L < 2 || q < 2 || q > 255 || nseqs == 0) return 0;
    const uint32_t nws[4] = {128, 256, 384, 512};
    for (uint32_t NW : nws) {
        if (nseqs % NW) continue;
        for (uint32_t S = 2; S <= 6; ++S) {
            // chunk sizes: stage buffers of about 8, 16, 24, 32, 48 KB
            const uint32_t kb[5] = {8, 16, 24, 32, 48};
            uint32_t last = 0;
            for (uint32_t t = 0; t < 5; ++t) {
                const uint32_t M = metro_chunk(L, q, kb[t] * 1024);
                if (M == last) continue;
                last = M;
                MetroConfig cfg;
                if (make_metro_config(L, q, nseqs, NW, M, S, cfg) != MI3_OK) continue;
                if (plans && n < max) {
                    plans[3 * n] = NW;
                    plans[3 * n + 1] = M;
                    plans[3 * n + 2] = S;
                }
                ++n;
            }
        }
    }
    set_error("");
    return n;
}

extern "C" int mi3_metropolis_plan(const float *Jrows, uint32_t *rngstates, uint32_t position_offset,
                                   const uint32_t *position_list, uint32_t nsteps, const float *betas,
                                   float beta, uint32_t *seqmem, uint32_t nseqs, uint32_t L, uint32_t q,
                                   uint32_t walkers_per_cta, uint32_t sites_per_chunk, uint32_t stages,
                                   int32_t *status, void *stream) {
    if (!Jrows || !rngstates || !position_list || !seqmem || !status)
        return fail(MI3_ERR_ARG, "mi3_metropolis: null pointer");
    if (L < 2 || q < 2 || q > 255) return fail(MI3_ERR_ARG, "mi3_metropolis: bad L/q");
    if (nseqs == 0 || nseqs % 128)
        return fail(MI3_ERR_ARG, "mi3_metropolis: nseqs must be a positive multiple of 128");
    if (!aligned(Jrows, 16) || !aligned(rngstates, 16))
        return fail(MI3_ERR_ALIGN, "mi3_metropolis: Jrows/rngstates must be 16B aligned");
    if (nsteps == 0) return MI3_OK;
    MetroConfig cfg;
    int rc = make_metro_config(L, q, nseqs, walkers_per_cta, sites_per_chunk, stages, cfg);
    if (rc) return rc;
    auto kernel = cfg.pk == 6 ? k_metropolis<6> : k_metropolis<4>;
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg.smem);
    MetroParams p;
    p.Jrows = Jrows;
    p.stride = jrow_stride(L, q);
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
    p.M = cfg.M;
    p.nchunks = cfg.nchunks;
    p.stages = cfg.stages;
    p.stage_floats = cfg.stage_floats;
    p.status = status;
    kernel<<<nseqs / cfg.NW, cfg.NW + 32, cfg.smem, as_stream(stream)>>>(p);
    return check_launch("mi3_metropolis");
}

extern "C" int mi3_metropolis(const float *Jrows, uint32_t *rngstates, uint32_t position_offset,
                              const uint32_t *position_list, uint32_t nsteps, const float *betas,
                              float beta, uint32_t *seqmem, uint32_t nseqs, uint32_t L, uint32_t q,
                              int32_t *status, void *stream) {
    return mi3_metropolis_plan(Jrows, rngstates, position_offset, position_list, nsteps, betas, beta, seqmem,
                               nseqs, L, q, 0, 0, 0, status, stream);
}
