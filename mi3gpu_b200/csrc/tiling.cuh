// tiling.cuh -- site-block tiling shared by the pair kernels (energies,
// bimarginal counts, weighted bimarginals).
//
// Sites are cut into blocks of B (a multiple of 4, so a block is B/4 whole
// sequence words).  A "slice" is a block pair (bi <= bj) and holds the
// B x B site pairs (i in bi, j in bj, i < j).  A CTA owns one slice (its
// couplings or its histograms stay in shared memory) and streams one chunk of
// sequences through it, reading only the 2*B/4 words of each sequence it
// needs.  Couplings are read once per (slice, chunk) and sequences once per
// slice, which keeps L2/HBM traffic far below the shared-memory work.
#pragma once
#include <algorithm>

#include "common.cuh"

namespace mi3 {

struct SliceGeom {
    uint32_t B;        // sites per block
    uint32_t nb;       // number of site blocks
    uint32_t nslices;  // nb*(nb+1)/2
    uint32_t chunk;    // sequences per CTA
    uint32_t nchunks;
};

// Slice index -> (bi, bj), row-major over the upper triangle including the
// diagonal.
__device__ __forceinline__ void slice_coords(uint32_t s, uint32_t nb, uint32_t &bi, uint32_t &bj) {
    uint32_t r = 0, base = 0;
    while (base + (nb - r) <= s) {
        base += nb - r;
        ++r;
    }
    bi = r;
    bj = r + (s - base);
}

__host__ __device__ __forceinline__ uint64_t pair_index(uint32_t i, uint32_t j, uint32_t L) {
    return (uint64_t)i * (2 * L - i - 1) / 2 + (j - i - 1);
}

// Largest block size whose slice of q*q-entry pairs fits in `budget` bytes.
inline uint32_t pick_block(uint32_t q, size_t budget) {
    const uint32_t cands[4] = {32, 16, 8, 4};
    for (uint32_t B : cands)
        if ((size_t)B * B * q * q * 4 <= budget) return B;
    return 0;
}

inline SliceGeom make_geom(uint32_t L, uint32_t B, uint32_t nseq, uint32_t target_ctas,
                           uint32_t min_chunk) {
    SliceGeom g;
    g.B = B;
    g.nb = (L + B - 1) / B;
    g.nslices = g.nb * (g.nb + 1) / 2;
    uint32_t want = std::max<uint32_t>(1, (target_ctas + g.nslices - 1) / g.nslices);
    uint32_t chunk = (nseq + want - 1) / want;
    chunk = std::max(chunk, min_chunk);
    chunk = (chunk + 255) & ~255u;
    g.chunk = chunk;
    g.nchunks = (nseq + chunk - 1) / chunk;
    return g;
}

// Load the B/4 words of block `b` of sequence n (zero past the last word).
template <int B>
__device__ __forceinline__ void load_block_words(const uint32_t *__restrict__ seq, uint32_t buflen,
                                                 uint32_t n, uint32_t b, uint32_t swords,
                                                 uint32_t (&w)[B / 4]) {
#pragma unroll
    for (int k = 0; k < B / 4; ++k) {
        uint32_t wi = b * (B / 4) + k;
        w[k] = (wi < swords) ? __ldg(&seq[(size_t)wi * buflen + n]) : 0u;
    }
}

// Residue k of a block, clamped to q-1: valid input never needs the clamp;
// it keeps shared-memory indexing in bounds for a corrupt residue byte.
template <int B>
__device__ __forceinline__ uint32_t block_byte(const uint32_t (&w)[B / 4], int k, uint32_t qm1) {
    return min((w[k >> 2] >> (8 * (k & 3))) & 0xffu, qm1);
}

}  // namespace mi3
