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

// Largest block size (at most max_b) whose slice of q*q-entry pairs fits in
// `budget` bytes.
inline uint32_t pick_block(uint32_t q, size_t budget, uint32_t max_b = 32) {
    const uint32_t cands[4] = {32, 16, 8, 4};
    for (uint32_t B : cands)
        if (B <= max_b && (size_t)B * B * q * q * 4 <= budget) return B;
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

// Fixed-point scale of the weighted histograms: increments are
// round(w * 2^s), with s chosen from the largest weight so that a whole
// chunk of `chunk` sequences fits a u32 bin:
// chunk * (wmax * 2^s + 1/2) <= 2^32 - 1.
__device__ __forceinline__ int fixed_shift(float wmax, uint32_t chunk) {
    if (!(wmax > 0.0f)) return 40;
    double lim = (4294967295.0 - (double)chunk) / ((double)chunk * (double)wmax);
    int s = (int)floor(log2(lim));
    return min(s, 40);
}

// The chunk length that sets that scale for mi3_weighted_marg on a shape
// (every weighted-histogram kernel uses it, so all give identical integers).
uint32_t wmarg_fixed_chunk(uint32_t L, uint32_t q, uint32_t nseq);

// Slice kinds: the B x B pairs of an off-diagonal block pair inside the
// sequence (every pair valid), a diagonal block pair inside the sequence
// (pairs jj > ii), and a block pair that crosses the end of the sequence
// (each pair tested).  Specialising on the kind removes the per-pair tests
// from the first two, which are all but a few slices.
enum SliceKind { SLICE_FULL = 0, SLICE_DIAG = 1, SLICE_EDGE = 2 };

__device__ __forceinline__ int slice_kind(uint32_t bi, uint32_t bj, uint32_t j0, uint32_t B, uint32_t L) {
    if (j0 + B > L) return SLICE_EDGE;
    return bi == bj ? SLICE_DIAG : SLICE_FULL;
}

// Whether pair (ii, jj) of a slice of kind K is a real pair i < j < L.
template <int K>
__device__ __forceinline__ bool slice_pair_valid(int ii, int jj, uint32_t i0, uint32_t j0, uint32_t L) {
    if constexpr (K == SLICE_FULL) return true;
    if constexpr (K == SLICE_DIAG) return jj > ii;
    return (j0 + jj < L) && (j0 + jj > i0 + ii);
}

// 32-bit shared-memory offsets of one sequence in a slice table laid out as
// [ii][jj][a][b]: col[jj] = jj*q*q + s_j, and the row of site ii is
// ii*B*q*q + s_i*q.
template <int B>
__device__ __forceinline__ void slice_cols(const uint32_t (&wJ)[B / 4], uint32_t q, uint32_t qq,
                                           uint32_t (&col)[B]) {
#pragma unroll
    for (int jj = 0; jj < B; ++jj) col[jj] = (uint32_t)jj * qq + block_byte<B>(wJ, jj, q - 1);
}

template <int B>
__device__ __forceinline__ uint32_t slice_row(const uint32_t (&wI)[B / 4], int ii, uint32_t q, uint32_t qq) {
    return (uint32_t)ii * B * qq + block_byte<B>(wI, ii, q - 1) * q;
}

// ------------------------------------------------ lanes over pairs (full slices)
// In a slice table laid out pair-major, [p][cell], the 32 sequences of a warp
// all visit pair p at the same time and gather 32 random cells: about 3.3
// shared-memory wavefronts per warp instruction.  For full slices (every
// pair valid) the pair kernels can instead lay the table out cell-major,
// [cell][p] with P = B*B pairs (p = ii*B + jj), and let lane w visit pair
// (t + w) mod P at step t: 32 consecutive pairs, 32 different banks, one
// wavefront.  Lane w = B*wh + wl then meets pair (ii, jj) with
// jj = (tl + wl) mod B and ii = (th + wh + carry) mod B for step
// t = B*th + tl, carry = (tl + wl >= B).  Rotating the sequence's residue
// bytes of block I by wh and of block J by wl (byte k of the rotated block
// = byte (k + r) mod B) turns these into static register indices: the
// column offset of step t is col[tl], the row offset row[th] or
// row[th + 1] -- one select per pair.  P >= 32 needs B >= 8.

// byte k of o = byte (k + r) mod B of w, for 0 <= r < B
template <int B>
__device__ __forceinline__ void rotate_block(const uint32_t (&w)[B / 4], uint32_t r, uint32_t (&o)[B / 4]) {
    constexpr int W = B / 4;
    const uint32_t rw = r >> 2, rb = 8 * (r & 3);
    uint32_t t[W];
#pragma unroll
    for (int k = 0; k < W; ++k) {
        uint32_t v = w[0];
#pragma unroll
        for (int j = 1; j < W; ++j) v = ((k + rw) % W == (uint32_t)j) ? w[j] : v;
        t[k] = v;
    }
#pragma unroll
    for (int k = 0; k < W; ++k) o[k] = __funnelshift_r(t[k], t[(k + 1) % W], rb);
}

// Byte offsets, in a [cell][P] float table, of lane's row (site ii of block
// I with residue a: a*q*P + ii*B) and column (site jj of block J with
// residue b: b*P + jj) terms, in rotated order.
template <int B>
__device__ __forceinline__ void lane_offsets(const uint32_t (&wI)[B / 4], const uint32_t (&wJ)[B / 4], uint32_t q,
                                             uint32_t lane, uint32_t (&row)[B], uint32_t (&col)[B]) {
    constexpr uint32_t P = B * B;
    const uint32_t wh = lane / B, wl = lane % B;
    uint32_t rI[B / 4], rJ[B / 4];
    rotate_block<B>(wI, wh, rI);
    rotate_block<B>(wJ, wl, rJ);
#pragma unroll
    for (int k = 0; k < B; ++k) {
        const uint32_t a = min((rI[k >> 2] >> (8 * (k & 3))) & 0xffu, q - 1);
        const uint32_t b = min((rJ[k >> 2] >> (8 * (k & 3))) & 0xffu, q - 1);
        row[k] = 4 * (a * q * P + ((k + wh) & (B - 1)) * B);
        col[k] = 4 * (b * P + ((k + wl) & (B - 1)));
    }
}

// ---------------------------------------------------------------- consensus
// Consensus decomposition.  Every site i has a reference residue c_i (any
// choice is exact; the most frequent residue makes it fastest).  A pair
// kernel then visits only the pairs where neither site holds its c:
//   - pair histograms: the bins of row c_i and column c_j are rebuilt
//     afterwards from per-site totals (integer arithmetic, exact);
//   - energies: couplings are first moved to the gauge where row c_i and
//     column c_j of every pair block are zero, the removed parts becoming
//     site fields and a constant.
// Consensus residues of block b packed like sequence words (byte k of word w
// is site b*B + 4w + k); 0xff past the last site.
template <int B>
__device__ __forceinline__ void load_cons_words(const uint8_t *__restrict__ cons, uint32_t b, uint32_t L,
                                                uint32_t (&c)[B / 4]) {
#pragma unroll
    for (int k = 0; k < B / 4; ++k) {
        uint32_t w = 0;
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            uint32_t site = b * B + 4 * k + t;
            uint32_t v = site < L ? (uint32_t)__ldg(&cons[site]) : 0xffu;
            w |= v << (8 * t);
        }
        c[k] = w;
    }
}

// Per-byte "residue differs from the consensus" masks (0xff / 0x00 bytes).
template <int B>
__device__ __forceinline__ void cons_masks(const uint32_t (&w)[B / 4], const uint32_t (&c)[B / 4],
                                           uint32_t (&m)[B / 4]) {
#pragma unroll
    for (int k = 0; k < B / 4; ++k) m[k] = __vcmpne4(w[k], c[k]);
}

template <int B>
__device__ __forceinline__ bool cons_off(const uint32_t (&m)[B / 4], int k) {
    return (m[k >> 2] >> (8 * (k & 3))) & 1u;
}

// Bit jj set when site jj of the block differs from its consensus.
template <int B>
__device__ __forceinline__ uint32_t cons_bits(const uint32_t (&m)[B / 4]) {
    uint32_t b = 0;
#pragma unroll
    for (int k = 0; k < B; ++k) b |= ((m[k >> 2] >> (8 * (k & 3))) & 1u) << k;
    return b;
}

// Predicated shared-memory access: one bit test selects the lanes, so the
// masked-off lanes cost no shared-memory bandwidth and no branch.
__device__ __forceinline__ float lds_if(uint32_t saddr, uint32_t bit) {
    float v;
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %2, 0;\n\tmov.f32 %0, 0f00000000;\n\t"
        "@p ld.shared.f32 %0, [%1];\n\t}"
        : "=f"(v)
        : "r"(saddr), "r"(bit));
    return v;
}

// (volatile asm keeps its order against the barriers around the pass; no
// memory clobber, so registers stay live across it)
__device__ __forceinline__ void red_add_if(uint32_t saddr, uint32_t inc, uint32_t bit) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %2, 0;\n\t@p red.shared.add.u32 [%0], %1;\n\t}" ::"r"(saddr),
        "r"(inc), "r"(bit));
}

}  // namespace mi3
