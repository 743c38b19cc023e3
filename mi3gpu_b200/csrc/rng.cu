// rng.cu -- MWC64X stream seeding (initRNG2) and independent-site sequence
// generation (gen_indep).
#include "common.cuh"

namespace mi3 {

constexpr uint64_t MWC_M = 18446383549859758079ull;  // A*2^32 - 1
constexpr uint64_t MWC_BASEID = 4077358422479273989ull;

// (a*b) mod M.  M = A*2^32 - 1, so 2^32*A == 1 (mod M): a 128-bit product
// hi*2^64 + lo reduces by folding.  Plain 128-bit remainder keeps it simple;
// this runs once per walker.
__device__ __forceinline__ uint64_t mulmod(uint64_t a, uint64_t b) {
    unsigned __int128 p = (unsigned __int128)a * b;
    return (uint64_t)(p % MWC_M);
}

__device__ uint64_t powmod(uint64_t a, uint64_t e) {
    uint64_t acc = 1, sq = a;
#pragma unroll 1
    while (e) {
        if (e & 1) acc = mulmod(acc, sq);
        sq = mulmod(sq, sq);
        e >>= 1;
    }
    return acc;
}

// State of the stream at distance `dist` from the generator's base point:
// x = BASEID * A^dist mod M, split as (x / A, x % A) -- the MWC64X seeding
// rule (skip_mwc.cl:58-76).
__device__ __forceinline__ void seed_at(uint64_t dist, uint32_t &x, uint32_t &c) {
    uint64_t v = mulmod(MWC_BASEID, powmod(MWC_A, dist));
    x = (uint32_t)(v / MWC_A);
    c = (uint32_t)(v % MWC_A);
}

__global__ void k_init_rng(uint4 *st, uint32_t n, uint64_t offset, uint64_t span) {
    uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    uint32_t x0, c0, x1, c1;
    seed_at(offset + (uint64_t(g) * 2 + 0) * span, x0, c0);
    seed_at(offset + (uint64_t(g) * 2 + 1) * span, x1, c1);
    st[g] = make_uint4(x0, x1, c0, c1);
}

// gen_indep: site `pos` of walker g takes the smallest residue r whose
// cumulative probability exceeds the uniform draw, by the reference's binary
// search; one vec2 draw serves two consecutive sites.
__global__ void k_gen_indep(uint32_t *seq, uint32_t buflen, uint32_t nseq, uint4 *st,
                            const float *__restrict__ cprob, uint32_t L, uint32_t q) {
    extern __shared__ float s_cprob[];  // (L, q-1)
    uint32_t ncp = L * (q - 1);
    for (uint32_t k = threadIdx.x; k < ncp; k += blockDim.x) s_cprob[k] = cprob[k];
    __syncthreads();
    uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nseq) return;
    uint4 s4 = st[g];
    Rng2 r{s4.x, s4.y, s4.z, s4.w};
    uint32_t r0 = 0, r1 = 0, word = 0;
    uint32_t pos;
    for (pos = 0; pos < L; pos++) {
        float u;
        if ((pos & 1) == 0) {
            rng_next2(r, r0, r1);
            u = uniform_map(r0);
        } else {
            u = uniform_map(r1);
        }
        const float *cp = s_cprob + pos * (q - 1);
        uint32_t bot = 0, mid;
        for (uint32_t span = q; span > 1; span -= mid) {
            mid = span / 2;
            if (u >= cp[bot + mid - 1]) bot += mid;
        }
        word = setbyte(word, pos & 3, bot);
        if (((pos + 1) & 3) == 0) {
            seq[(size_t)(pos >> 2) * buflen + g] = word;
            word = 0;
        }
    }
    if (pos & 3) seq[(size_t)(pos >> 2) * buflen + g] = word;
    st[g] = make_uint4(r.x0, r.x1, r.c0, r.c1);
}

}  // namespace mi3

using namespace mi3;

extern "C" int mi3_init_rng(uint32_t *rngstates, uint32_t nwalkers, uint64_t rng_offset,
                            uint64_t walker_span, void *stream) {
    if (!rngstates || nwalkers == 0) return fail(MI3_ERR_ARG, "mi3_init_rng: null or empty");
    if (!aligned(rngstates, 16)) return fail(MI3_ERR_ALIGN, "mi3_init_rng: rngstates not 16B aligned");
    uint32_t tb = 128;
    k_init_rng<<<(nwalkers + tb - 1) / tb, tb, 0, as_stream(stream)>>>(
        reinterpret_cast<uint4 *>(rngstates), nwalkers, rng_offset, walker_span);
    return check_launch("mi3_init_rng");
}

extern "C" int mi3_gen_indep(uint32_t *seqmem, uint32_t buflen, uint32_t nseq, uint32_t *rngstates,
                             const float *cprob, uint32_t L, uint32_t q, void *stream) {
    if (!seqmem || !rngstates || !cprob) return fail(MI3_ERR_ARG, "mi3_gen_indep: null pointer");
    if (L < 2 || q < 2 || q > 255 || nseq == 0 || nseq > buflen)
        return fail(MI3_ERR_ARG, "mi3_gen_indep: bad L/q/nseq");
    size_t smem = sizeof(float) * L * (q - 1);
    if (smem > 200 * 1024) return fail(MI3_ERR_ARG, "mi3_gen_indep: L*(q-1) too large");
    if (!aligned(rngstates, 16)) return fail(MI3_ERR_ALIGN, "mi3_gen_indep: rngstates alignment");
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(k_gen_indep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    uint32_t tb = 256;
    k_gen_indep<<<(nseq + tb - 1) / tb, tb, smem, as_stream(stream)>>>(
        seqmem, buflen, nseq, reinterpret_cast<uint4 *>(rngstates), cprob, L, q);
    return check_launch("mi3_gen_indep");
}
