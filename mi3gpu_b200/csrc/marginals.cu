// marginals.cu -- pair histograms of the walkers' sequences.
//
//   mi3_bicounts        exact uint32 counts (countBivariate, mcmc.cl:462-516)
//   mi3_weighted_marg   weighted sums (weightedMarg, mcmc.cl:646-718), fixed point
//   mi3_bicounts_to_bimarg, mi3_renormalize_bimarg, mi3_repack_seqs_T
//
// The histogram kernels use the slice tiling of tiling.cuh: a CTA keeps the
// B*B pair histograms (q*q bins each) of one block pair in shared memory,
// increments them with shared-memory atomics for a chunk of sequences, and
// flushes them once.  Counts are integers, so they are exact whatever the
// order.
#include "tiling.cuh"

namespace mi3 {

// Pair histograms over a chunk of sequences, two sequences per thread (two
// independent atomic streams in flight).  WEIGHTED=false: +1 per sequence
// (exact counts, flushed as u32).  WEIGHTED=true: +round(w * 2^s) per
// sequence in u32 fixed point; s is chosen from the largest weight so a CTA's
// bin cannot overflow, and the CTA flushes into a u64 accumulator with
// integer atomics -- the sums are exact integers, so the result does not
// depend on the order of the atomics (deterministic).
// Increments of one sequence into the slice's histograms.  CONS: only the
// pairs where neither residue is its site's consensus (the others are
// rebuilt from site totals after the pass).
template <int B, int K, bool CONS, bool ROT>
__device__ __forceinline__ void slice_hist(uint32_t *h, const uint32_t (&wI)[B / 4], const uint32_t (&wJ)[B / 4],
                                           const uint32_t (&cI)[B / 4], const uint32_t (&cJ)[B / 4],
                                           uint32_t inc, uint32_t q, uint32_t qq, uint32_t i0, uint32_t j0,
                                           uint32_t L) {
    uint32_t col[B];
    if constexpr (ROT && !CONS && K == SLICE_FULL) {
        // Column order rotated by lane: at step t lane l updates column
        // (t + l) mod B, so one warp instruction spreads over B pair tables
        // and lanes rarely hit the same bin (same-bin lanes with different
        // increments are serialised by the shared-memory atomic unit; equal
        // increments, as in plain counts, are not, so counts keep the
        // unrotated order, which has fewer bank conflicts).
        const uint32_t rot = threadIdx.x & (B - 1);
#pragma unroll
        for (int t = 0; t < B; ++t) {
            const uint32_t jj = (t + rot) & (B - 1);
            uint32_t w = wJ[0];
#pragma unroll
            for (int k = 1; k < B / 4; ++k) w = ((jj >> 2) == (uint32_t)k) ? wJ[k] : w;
            col[t] = jj * qq + min((w >> (8 * (jj & 3))) & 0xffu, q - 1);
        }
#pragma unroll
        for (int ii = 0; ii < B; ++ii) {
            const uint32_t row = slice_row<B>(wI, ii, q, qq);
#pragma unroll
            for (int t = 0; t < B; ++t) atomicAdd(&h[row + col[t]], inc);
        }
        return;
    }
    slice_cols<B>(wJ, q, qq, col);
    if constexpr (!CONS) {
#pragma unroll
        for (int ii = 0; ii < B; ++ii) {
            if (K == SLICE_EDGE && i0 + ii >= L) break;
            const uint32_t row = slice_row<B>(wI, ii, q, qq);
#pragma unroll
            for (int jj = 0; jj < B; ++jj)
                if (slice_pair_valid<K>(ii, jj, i0, j0, L)) atomicAdd(&h[row + col[jj]], inc);
        }
    } else {
        uint32_t mI[B / 4], mJ[B / 4];
        cons_masks<B>(wI, cI, mI);
        cons_masks<B>(wJ, cJ, mJ);
        const uint32_t cb = cons_bits<B>(mJ);
        const uint32_t base = (uint32_t)__cvta_generic_to_shared(h);
#pragma unroll
        for (int ii = 0; ii < B; ++ii) {
            if (K == SLICE_EDGE && i0 + ii >= L) break;
            const uint32_t row = slice_row<B>(wI, ii, q, qq);
            const uint32_t rb = cons_off<B>(mI, ii) ? cb : 0u;  // active columns of this row
#pragma unroll
            for (int jj = 0; jj < B; ++jj)
                if (slice_pair_valid<K>(ii, jj, i0, j0, L)) red_add_if(base + 4u * (row + col[jj]), inc, rb & (1u << jj));
        }
    }
}

template <int B, int K, bool WEIGHTED, bool CONS>
__device__ __forceinline__ void hist_chunk(uint32_t *h, const uint32_t *__restrict__ seq, uint32_t buflen,
                                           uint32_t nbeg, uint32_t nend, const float *__restrict__ weights,
                                           float scale, uint32_t L, uint32_t q, uint32_t bi, uint32_t bj,
                                           const uint32_t (&cI)[B / 4], const uint32_t (&cJ)[B / 4]) {
    const uint32_t qq = q * q, swords = (L - 1) / 4 + 1;
    const uint32_t i0 = bi * B, j0 = bj * B;
    if constexpr (B == 16 && CONS) {
        // 16-site blocks with consensus masks: one sequence per thread keeps
        // the offsets and masks in registers
        for (uint32_t n = nbeg + threadIdx.x; n < nend; n += blockDim.x) {
            uint32_t wI[B / 4], wJ[B / 4];
            load_block_words<B>(seq, buflen, n, bi, swords, wI);
            load_block_words<B>(seq, buflen, n, bj, swords, wJ);
            uint32_t inc = 1u;
            if constexpr (WEIGHTED) inc = __float2uint_rn(__ldg(&weights[n]) * scale);
            slice_hist<B, K, CONS, false>(h, wI, wJ, cI, cJ, inc, q, qq, i0, j0, L);
        }
    } else {
        // two sequences per thread: two independent atomic streams in flight
        for (uint32_t n = nbeg + threadIdx.x; n < nend; n += 2 * blockDim.x) {
            const uint32_t n2 = n + blockDim.x;
            const bool two = n2 < nend;
            uint32_t wI[B / 4], wJ[B / 4], vI[B / 4], vJ[B / 4];
            load_block_words<B>(seq, buflen, n, bi, swords, wI);
            load_block_words<B>(seq, buflen, n, bj, swords, wJ);
            load_block_words<B>(seq, buflen, two ? n2 : n, bi, swords, vI);
            load_block_words<B>(seq, buflen, two ? n2 : n, bj, swords, vJ);
            uint32_t inc1 = 1u, inc2 = 1u;
            if constexpr (WEIGHTED) {
                inc1 = __float2uint_rn(__ldg(&weights[n]) * scale);
                inc2 = two ? __float2uint_rn(__ldg(&weights[n2]) * scale) : 0u;
            }
            constexpr bool ROT = WEIGHTED && B <= 8;
            slice_hist<B, K, CONS, ROT>(h, wI, wJ, cI, cJ, inc1, q, qq, i0, j0, L);
            if (two) slice_hist<B, K, CONS, ROT>(h, vI, vJ, cI, cJ, inc2, q, qq, i0, j0, L);
        }
    }
}

// Full slices with lanes over pairs (tiling.cuh): the histograms are
// [cell][P]; lane w adds to pair (t + w) mod P at step t, so the 32 lanes of
// a shared-memory reduction always hit 32 different banks and different
// bins (no serialised same-bin adds either).
template <int B>
__device__ __forceinline__ void lane_hist(uint32_t hbase, const uint32_t (&row)[B], const uint32_t (&col)[B],
                                          uint32_t wl, uint32_t inc) {
#pragma unroll
    for (int tl = 0; tl < B; ++tl) {
        const bool carry = tl + wl >= (uint32_t)B;
        const uint32_t c = hbase + col[tl];
#pragma unroll
        for (int th = 0; th < B; ++th) {
            const uint32_t r = carry ? row[(th + 1) & (B - 1)] : row[th];
            asm volatile("red.shared.add.u32 [%0], %1;" ::"r"(c + r), "r"(inc));
        }
    }
}

template <int B, bool WEIGHTED>
__device__ __forceinline__ void hist_chunk_lanes(uint32_t *h, const uint32_t *__restrict__ seq, uint32_t buflen,
                                                 uint32_t nbeg, uint32_t nend, const float *__restrict__ weights,
                                                 float scale, uint32_t L, uint32_t q, uint32_t bi, uint32_t bj) {
    const uint32_t swords = (L - 1) / 4 + 1;
    const uint32_t lane = threadIdx.x & 31, wl = lane % B;
    const uint32_t hbase = (uint32_t)__cvta_generic_to_shared(h);
    if constexpr (B == 16) {
        for (uint32_t n = nbeg + threadIdx.x; n < nend; n += blockDim.x) {
            uint32_t wI[B / 4], wJ[B / 4];
            load_block_words<B>(seq, buflen, n, bi, swords, wI);
            load_block_words<B>(seq, buflen, n, bj, swords, wJ);
            uint32_t inc = 1u;
            if constexpr (WEIGHTED) inc = __float2uint_rn(__ldg(&weights[n]) * scale);
            uint32_t row[B], col[B];
            lane_offsets<B>(wI, wJ, q, lane, row, col);
            lane_hist<B>(hbase, row, col, wl, inc);
        }
        return;
    }
    for (uint32_t n = nbeg + threadIdx.x; n < nend; n += 2 * blockDim.x) {
        const uint32_t n2 = n + blockDim.x;
        const bool two = n2 < nend;
        uint32_t wI[B / 4], wJ[B / 4], vI[B / 4], vJ[B / 4];
        load_block_words<B>(seq, buflen, n, bi, swords, wI);
        load_block_words<B>(seq, buflen, n, bj, swords, wJ);
        load_block_words<B>(seq, buflen, two ? n2 : n, bi, swords, vI);
        load_block_words<B>(seq, buflen, two ? n2 : n, bj, swords, vJ);
        uint32_t inc1 = 1u, inc2 = 1u;
        if constexpr (WEIGHTED) {
            inc1 = __float2uint_rn(__ldg(&weights[n]) * scale);
            inc2 = two ? __float2uint_rn(__ldg(&weights[n2]) * scale) : 0u;
        }
        uint32_t row[B], col[B];
        lane_offsets<B>(wI, wJ, q, lane, row, col);
        lane_hist<B>(hbase, row, col, wl, inc1);
        lane_offsets<B>(vI, vJ, q, lane, row, col);
        lane_hist<B>(hbase, row, col, wl, two ? inc2 : 0u);
    }
}

template <int B, bool WEIGHTED, bool CONS>
__global__ void __launch_bounds__(512, 2) k_pairhist(const uint32_t *__restrict__ seq, uint32_t buflen,
                                                     uint32_t nseq, const float *__restrict__ weights,
                                                     const unsigned int *__restrict__ wmax_bits, void *out,
                                                     uint32_t L, uint32_t q, SliceGeom g, uint64_t nbins,
                                                     const uint8_t *__restrict__ cons) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint32_t *h = reinterpret_cast<uint32_t *>(smem_raw);  // [B*B][q*q]
    const uint32_t qq = q * q;
    const uint32_t s = blockIdx.x % g.nslices;
    const uint32_t chunk = blockIdx.x / g.nslices;
    uint32_t bi, bj;
    slice_coords(s, g.nb, bi, bj);
    const uint32_t i0 = bi * B, j0 = bj * B;
    const uint32_t nh = B * B * qq;
    for (uint32_t k = threadIdx.x; k < nh; k += blockDim.x) h[k] = 0u;
    float scale = 1.0f;
    if constexpr (WEIGHTED) scale = ldexpf(1.0f, fixed_shift(__uint_as_float(*wmax_bits), g.chunk));
    uint32_t cI[B / 4] = {}, cJ[B / 4] = {};
    if constexpr (CONS) {
        load_cons_words<B>(cons, bi, L, cI);
        load_cons_words<B>(cons, bj, L, cJ);
    }
    __syncthreads();

    const uint32_t nbeg = chunk * g.chunk;
    const uint32_t nend = min(nseq, nbeg + g.chunk);
    const int kind = slice_kind(bi, bj, j0, B, L);
    if constexpr (!CONS && B >= 8) {
        if (kind == SLICE_FULL) {
            hist_chunk_lanes<B, WEIGHTED>(h, seq, buflen, nbeg, nend, weights, scale, L, q, bi, bj);
            __syncthreads();
            // flush the [cell][P] table: lane l takes cell c0 + l % 8 of pair
            // p0 + l / 8 -- global writes of 8 consecutive cells of 4 pairs
            constexpr uint32_t P = B * B;
            const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
            const uint32_t cgroups = (qq + 7) / 8;
            for (uint32_t t = warp; t < cgroups * (P / 4); t += nwarps) {
                const uint32_t c = (t % cgroups) * 8 + (lane & 7), p = (t / cgroups) * 4 + (lane >> 3);
                if (c >= qq) continue;
                const uint32_t v = h[c * P + p];
                const uint64_t dst = pair_index(i0 + p / B, j0 + p % B, L) * qq + c;
                if constexpr (WEIGHTED) {
                    reinterpret_cast<uint32_t *>(out)[(uint64_t)chunk * nbins + dst] = v;
                } else if (g.nchunks > 1) {
                    if (v) atomicAdd(reinterpret_cast<uint32_t *>(out) + dst, v);
                } else {
                    reinterpret_cast<uint32_t *>(out)[dst] = v;
                }
            }
            return;
        }
    }
    switch (kind) {
        case SLICE_FULL:
            hist_chunk<B, SLICE_FULL, WEIGHTED, CONS>(h, seq, buflen, nbeg, nend, weights, scale, L, q, bi, bj,
                                                      cI, cJ);
            break;
        case SLICE_DIAG:
            hist_chunk<B, SLICE_DIAG, WEIGHTED, CONS>(h, seq, buflen, nbeg, nend, weights, scale, L, q, bi, bj,
                                                      cI, cJ);
            break;
        default:
            hist_chunk<B, SLICE_EDGE, WEIGHTED, CONS>(h, seq, buflen, nbeg, nend, weights, scale, L, q, bi, bj,
                                                      cI, cJ);
            break;
    }
    __syncthreads();
    // flush the slice's valid pairs
    for (int ii = 0; ii < B; ++ii) {
        uint32_t i = i0 + ii;
        if (i + 1 >= L) break;
        uint32_t jlo = max(j0, i + 1), jhi = min(j0 + B, L);
        if (jlo >= jhi) continue;
        const uint64_t dst0 = pair_index(i, jlo, L) * qq;
        const uint32_t *src = h + ((size_t)ii * B + (jlo - j0)) * qq;
        uint32_t cnt = (jhi - jlo) * qq;
        for (uint32_t k = threadIdx.x; k < cnt; k += blockDim.x) {
            uint32_t v = src[k];
            if constexpr (WEIGHTED) {
                // this chunk's partial sums: a plain store into its own plane
                reinterpret_cast<uint32_t *>(out)[(uint64_t)chunk * nbins + dst0 + k] = v;
            } else if (g.nchunks > 1) {
                if (v) atomicAdd(reinterpret_cast<uint32_t *>(out) + dst0 + k, v);
            } else {
                reinterpret_cast<uint32_t *>(out)[dst0 + k] = v;
            }
        }
    }
}

// Largest weight (weights are >= 0, so the float order is the bit order).
__global__ void k_wmax(const float *__restrict__ w, uint32_t n, unsigned int *out) {
    float m = 0.0f;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        m = fmaxf(m, w[k]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m > 0.0f) atomicMax(out, __float_as_uint(m));
}

// Per-chunk fixed-point partial sums -> float weighted bimarginals: each bin
// sums its nchunks partials in a fixed order (exact integers), then scales.
__global__ void k_chunks_to_float(const uint32_t *__restrict__ part, uint32_t nchunks,
                                  const unsigned int *wmax_bits, uint32_t chunk, float *out, uint64_t n) {
    uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    unsigned long long acc = 0;
    for (uint32_t c = 0; c < nchunks; ++c) acc += __ldg(&part[(uint64_t)c * n + k]);
    int s = fixed_shift(__uint_as_float(*wmax_bits), chunk);
    out[k] = (float)ldexp((double)acc, -s);
}

constexpr uint32_t WMARG_CHUNK = 65536;  // sequences per CTA (fixed-point headroom)

template <int B, bool WEIGHTED>
static SliceGeom pairhist_geom(uint32_t L, uint32_t nseq) {
    SliceGeom g = make_geom(L, B, nseq, 148 * 8, 2048);
    if (WEIGHTED && g.chunk > WMARG_CHUNK) {
        g.chunk = WMARG_CHUNK;
        g.nchunks = (nseq + g.chunk - 1) / g.chunk;
    }
    return g;
}

// Per-site residue sums over blocks of at most per_cta sequences (<= the pair
// kernel's chunk, so the same fixed-point increments fit u32 bins):
// WEIGHTED adds the pair kernel's rounded weight, else 1.  CONS skips each
// site's consensus residue (the rebuild does not need it).  usite (u64,
// L x q) and *wtot (the sum of all increments) are accumulated with integer
// atomics, so they are exact.
template <bool WEIGHTED, bool CONS>
__global__ void __launch_bounds__(256) k_site_hist(const uint32_t *__restrict__ seq, uint32_t buflen,
                                                   uint32_t nseq, const float *__restrict__ weights,
                                                   const unsigned int *__restrict__ wmax_bits,
                                                   uint32_t fix_chunk, const uint8_t *__restrict__ cons,
                                                   unsigned long long *usite, unsigned long long *wtot,
                                                   uint32_t L, uint32_t q, uint32_t per_cta) {
    extern __shared__ uint32_t sh[];  // [L*q] bins, then L consensus bytes
    uint8_t *sc = reinterpret_cast<uint8_t *>(sh + L * q);
    __shared__ unsigned long long red[8];
    for (uint32_t k = threadIdx.x; k < L * q; k += blockDim.x) sh[k] = 0u;
    if constexpr (CONS)
        for (uint32_t k = threadIdx.x; k < L; k += blockDim.x) sc[k] = cons[k];
    float scale = 1.0f;
    if constexpr (WEIGHTED) scale = ldexpf(1.0f, fixed_shift(__uint_as_float(*wmax_bits), fix_chunk));
    __syncthreads();
    const uint32_t swords = (L - 1) / 4 + 1;
    const uint32_t beg = blockIdx.x * per_cta, end = min(nseq, beg + per_cta);
    unsigned long long mine = 0;
    for (uint32_t n = beg + threadIdx.x; n < end; n += blockDim.x) {
        uint32_t inc = 1u;
        if constexpr (WEIGHTED) inc = __float2uint_rn(__ldg(&weights[n]) * scale);
        mine += inc;
        for (uint32_t wd = 0; wd < swords; ++wd) {
            const uint32_t word = __ldg(&seq[(size_t)wd * buflen + n]);
#pragma unroll
            for (uint32_t t = 0; t < 4; ++t) {
                const uint32_t site = 4 * wd + t;
                const uint32_t a = min((word >> (8 * t)) & 0xffu, q - 1);
                if (site < L && (!CONS || a != sc[site])) atomicAdd(&sh[site * q + a], inc);
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) mine += __shfl_down_sync(0xffffffffu, mine, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mine;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (uint32_t k = 0; k < (blockDim.x >> 5); ++k) t += red[k];
        if (wtot) atomicAdd(wtot, t);
    }
    for (uint32_t k = threadIdx.x; k < L * q; k += blockDim.x)
        if (sh[k]) atomicAdd(&usite[k], (unsigned long long)sh[k]);
}

// Most frequent residue of every site (the lowest on ties).
__global__ void k_argmax_sites(const unsigned long long *__restrict__ cnt, uint8_t *cons, uint32_t L, uint32_t q) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L) return;
    uint32_t best = 0;
    unsigned long long bv = cnt[(size_t)i * q];
    for (uint32_t a = 1; a < q; ++a) {
        const unsigned long long v = cnt[(size_t)i * q + a];
        if (v > bv) {
            bv = v;
            best = a;
        }
    }
    cons[i] = (uint8_t)best;
}

// Per-chunk planes of the non-consensus pair bins -> all bins of every pair:
// sum the planes, rebuild row c_i and column c_j from the site totals,
// the corner from the total, and scale to float.  Integer arithmetic
// throughout: the bins equal those of a direct count with the same
// increments.  One CTA per pair; tile of q*q u64 in shared memory.
__global__ void __launch_bounds__(128) k_pairs_rebuild(const uint32_t *__restrict__ part, uint32_t nchunks,
                                                       const unsigned long long *__restrict__ usite,
                                                       const unsigned long long *__restrict__ wtot,
                                                       const unsigned int *__restrict__ wmax_bits,
                                                       uint32_t fix_chunk, const uint8_t *__restrict__ cons,
                                                       float *out, uint32_t L, uint32_t q, uint64_t nbins) {
    extern __shared__ unsigned long long tile[];  // [q*q]
    __shared__ uint32_t ij[2];
    const uint32_t p = blockIdx.x, qq = q * q;
    if (threadIdx.x == 0) {
        uint32_t r = 0;
        uint64_t start = 0;
        while (r + 1 < L && p >= start + (L - 1 - r)) {
            start += L - 1 - r;
            ++r;
        }
        ij[0] = r;
        ij[1] = r + 1 + (uint32_t)(p - start);
    }
    for (uint32_t e = threadIdx.x; e < qq; e += blockDim.x) {
        unsigned long long acc = 0;
        for (uint32_t c = 0; c < nchunks; ++c) acc += __ldg(&part[(uint64_t)c * nbins + (uint64_t)p * qq + e]);
        tile[e] = acc;
    }
    __syncthreads();
    const uint32_t i = ij[0], j = ij[1];
    const uint32_t ci = min((uint32_t)cons[i], q - 1), cj = min((uint32_t)cons[j], q - 1);
    const unsigned long long *ui = usite + (size_t)i * q, *uj = usite + (size_t)j * q;
    // column c_j of rows a != c_i, and row c_i of columns b != c_j
    for (uint32_t t = threadIdx.x; t < 2 * q; t += blockDim.x) {
        if (t < q) {
            const uint32_t a = t;
            if (a == ci) continue;
            unsigned long long r = 0;
            for (uint32_t b = 0; b < q; ++b)
                if (b != cj) r += tile[a * q + b];
            tile[a * q + cj] = ui[a] - r;
        } else {
            const uint32_t b = t - q;
            if (b == cj) continue;
            unsigned long long c = 0;
            for (uint32_t a = 0; a < q; ++a)
                if (a != ci) c += tile[a * q + b];
            tile[ci * q + b] = uj[b] - c;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        // site i's consensus total is W minus its other residues; the corner
        // is that total minus the rest of row c_i
        unsigned long long rowc = *wtot;
        for (uint32_t a = 0; a < q; ++a)
            if (a != ci) rowc -= ui[a];
        for (uint32_t b = 0; b < q; ++b)
            if (b != cj) rowc -= tile[ci * q + b];
        tile[ci * q + cj] = rowc;
    }
    __syncthreads();
    const int s = fixed_shift(__uint_as_float(*wmax_bits), fix_chunk);
    for (uint32_t e = threadIdx.x; e < qq; e += blockDim.x)
        out[(uint64_t)p * qq + e] = (float)ldexp((double)tile[e], -s);
}

// Workspace of the weighted histograms: [wmax u32 | pad | wtot u64 | pad to
// 256][usite L*q u64, padded to 256][nchunks planes of nbins u32].
struct WmargWs {
    unsigned int *wmax;
    unsigned long long *wtot;
    unsigned long long *usite;
    uint32_t *planes;
};

inline size_t usite_bytes(uint32_t L, uint32_t q) { return ((size_t)L * q * 8 + 255) & ~size_t(255); }

inline WmargWs wmarg_ws(unsigned char *ws, uint32_t L, uint32_t q) {
    WmargWs w;
    w.wmax = reinterpret_cast<unsigned int *>(ws);
    w.wtot = reinterpret_cast<unsigned long long *>(ws + 8);
    w.usite = reinterpret_cast<unsigned long long *>(ws + 256);
    w.planes = reinterpret_cast<uint32_t *>(ws + 256 + usite_bytes(L, q));
    return w;
}

// Shapes the consensus rebuild handles: the q*q tile and the site histogram
// must fit shared memory.
inline bool cons_supported(uint32_t L, uint32_t q) {
    return q <= 64 && ((size_t)L * q * 4 + L) <= 160 * 1024;
}

template <int B, bool WEIGHTED, bool CONS>
static int launch_pairhist(const uint32_t *seq, uint32_t buflen, uint32_t nseq, const float *w,
                           unsigned char *ws, void *out, uint32_t L, uint32_t q, const uint8_t *cons,
                           cudaStream_t st) {
    SliceGeom g = pairhist_geom<B, WEIGHTED>(L, nseq);
    size_t smem = (size_t)B * B * q * q * 4;
    cudaFuncSetAttribute(k_pairhist<B, WEIGHTED, CONS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    uint64_t nblk = (uint64_t)g.nslices * g.nchunks;
    if (nblk > 0x7fffffffull) return fail(MI3_ERR_ARG, "pair histogram: grid too large");
    const uint64_t nbins = npairs_of(L) * q * q;
    if (!WEIGHTED) {
        if (g.nchunks > 1 && cudaMemsetAsync(out, 0, nbins * 4, st) != cudaSuccess)
            return check_launch("bicounts: memset");
        k_pairhist<B, false, false><<<(uint32_t)nblk, 512, smem, st>>>(seq, buflen, nseq, w, nullptr, out, L, q, g,
                                                                      nbins, nullptr);
        return check_launch("mi3_bicounts");
    }
    // every bin of every chunk plane is stored by the kernel: only the
    // scalars and the site totals need clearing
    WmargWs W = wmarg_ws(ws, L, q);
    if (cudaMemsetAsync(ws, 0, 256 + (CONS ? usite_bytes(L, q) : 0), st) != cudaSuccess)
        return check_launch("weighted marg: memset");
    k_wmax<<<296, 512, 0, st>>>(w, nseq, W.wmax);
    k_pairhist<B, true, CONS><<<(uint32_t)nblk, 512, smem, st>>>(seq, buflen, nseq, w, W.wmax, W.planes, L, q, g,
                                                                nbins, cons);
    int rc = check_launch("mi3_weighted_marg");
    if (rc) return rc;
    if (!CONS) {
        k_chunks_to_float<<<(uint32_t)((nbins + 255) / 256), 256, 0, st>>>(W.planes, g.nchunks, W.wmax, g.chunk,
                                                                          reinterpret_cast<float *>(out), nbins);
        return check_launch("mi3_weighted_marg: planes");
    }
    const uint32_t per_cta = std::min<uint32_t>(g.chunk, std::max<uint32_t>(256, (nseq + 148 * 4 - 1) / (148 * 4)));
    const size_t ssm = (size_t)L * q * 4 + L;
    if (ssm > 48 * 1024)
        cudaFuncSetAttribute(k_site_hist<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ssm);
    k_site_hist<true, true><<<(nseq + per_cta - 1) / per_cta, 256, ssm, st>>>(
        seq, buflen, nseq, w, W.wmax, g.chunk, cons, W.usite, W.wtot, L, q, per_cta);
    rc = check_launch("mi3_weighted_marg: sites");
    if (rc) return rc;
    k_pairs_rebuild<<<(uint32_t)npairs_of(L), 128, (size_t)q * q * 8, st>>>(
        W.planes, g.nchunks, W.usite, W.wtot, W.wmax, g.chunk, cons, reinterpret_cast<float *>(out), L, q, nbins);
    return check_launch("mi3_weighted_marg: rebuild");
}

template <bool WEIGHTED>
static int dispatch_pairhist(const uint32_t *seq, uint32_t buflen, uint32_t nseq, const float *w,
                             unsigned char *ws, void *out, uint32_t L, uint32_t q, const uint8_t *cons,
                             cudaStream_t st) {
    const uint32_t B = pick_block(q, 116 * 1024, 16);
    if constexpr (WEIGHTED) {
        if (cons != nullptr && cons_supported(L, q)) {
            switch (B) {
                case 16: return launch_pairhist<16, true, true>(seq, buflen, nseq, w, ws, out, L, q, cons, st);
                case 8: return launch_pairhist<8, true, true>(seq, buflen, nseq, w, ws, out, L, q, cons, st);
                case 4: return launch_pairhist<4, true, true>(seq, buflen, nseq, w, ws, out, L, q, cons, st);
                default: break;
            }
        }
    }
    switch (B) {
        case 16: return launch_pairhist<16, WEIGHTED, false>(seq, buflen, nseq, w, ws, out, L, q, nullptr, st);
        case 8: return launch_pairhist<8, WEIGHTED, false>(seq, buflen, nseq, w, ws, out, L, q, nullptr, st);
        case 4: return launch_pairhist<4, WEIGHTED, false>(seq, buflen, nseq, w, ws, out, L, q, nullptr, st);
        default: return fail(MI3_ERR_ARG, "pair histogram: q too large");
    }
}

__global__ void k_bicounts_to_bimarg(const uint32_t *__restrict__ c, float *bi, float nseq, uint64_t n) {
    uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) bi[k] = ((float)c[k]) / nseq;
}

// One warp per pair; the q*q row sum follows the reference's odd-aware tree
// (sumqq, mcmc.cl:732-751) so the normalised values agree bit for bit.
__global__ void k_renormalize(float *bi, uint64_t npairs, uint32_t qq) {
    extern __shared__ float sc_all[];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float *sc = sc_all + warp * qq;
    const uint32_t wpb = blockDim.x >> 5;
    for (uint64_t p = (uint64_t)blockIdx.x * wpb + warp; p < npairs; p += (uint64_t)gridDim.x * wpb) {
        float *row = bi + p * qq;
        for (uint32_t li = lane; li < qq; li += 32) sc[li] = row[li];
        __syncwarp();
        uint32_t m = qq;
        while (m > 1) {
            uint32_t odd = m & 1;
            m = (m + 1) >> 1;
            for (uint32_t li = lane; li < m - odd; li += 32) sc[li] = sc[li] + sc[li + m];
            __syncwarp();
        }
        float tot = sc[0];
        __syncwarp();
        for (uint32_t li = lane; li < qq; li += 32) row[li] = row[li] / tot;
        __syncwarp();
    }
}

// (SWORDS, buf4len) words -> byte matrix (L, 4*buf1len): row i holds site i
// of every sequence (the transpose of the host (N, L) array).
__global__ void k_repack_T(const uint32_t *__restrict__ seq4, uint32_t buf4len, uint32_t *seqL,
                           uint32_t buf1len, uint32_t L) {
    uint32_t i = blockIdx.y;
    uint32_t n4 = blockIdx.x * blockDim.x + threadIdx.x;
    if (n4 >= buf1len) return;
    uint32_t out = 0;
#pragma unroll
    for (uint32_t k = 0; k < 4; ++k) {
        uint32_t n = 4 * n4 + k;
        uint32_t b = (n < buf4len) ? getbyte(seq4[(size_t)(i >> 2) * buf4len + n], i & 3) : 0u;
        out |= b << (8 * k);
    }
    seqL[(size_t)i * buf1len + n4] = out;
}

}  // namespace mi3

using namespace mi3;

extern "C" int mi3_bicounts(const uint32_t *seqmem, uint32_t buflen, uint32_t nseq, uint32_t *bicount,
                            uint32_t L, uint32_t q, void *stream) {
    if (!seqmem || !bicount) return fail(MI3_ERR_ARG, "mi3_bicounts: null pointer");
    if (L < 2 || q < 1 || q > 255 || nseq > buflen) return fail(MI3_ERR_ARG, "mi3_bicounts: bad L/q/nseq");
    if (nseq == 0) {
        cudaMemsetAsync(bicount, 0, (size_t)npairs_of(L) * q * q * 4, as_stream(stream));
        return check_launch("mi3_bicounts: memset");
    }
    return dispatch_pairhist<false>(seqmem, buflen, nseq, nullptr, nullptr, bicount, L, q, nullptr,
                                    as_stream(stream));
}

namespace mi3 {
uint32_t wmarg_fixed_chunk(uint32_t L, uint32_t q, uint32_t nseq) {
    switch (pick_block(q, 116 * 1024, 16)) {
        case 16: return pairhist_geom<16, true>(L, nseq).chunk;
        case 8: return pairhist_geom<8, true>(L, nseq).chunk;
        case 4: return pairhist_geom<4, true>(L, nseq).chunk;
        default: return WMARG_CHUNK;
    }
}
}  // namespace mi3

extern "C" size_t mi3_weighted_marg_workspace(uint32_t L, uint32_t q, uint32_t nseq) {
    uint32_t nchunks = 1;
    switch (pick_block(q, 116 * 1024, 16)) {
        case 16: nchunks = pairhist_geom<16, true>(L, nseq).nchunks; break;
        case 8: nchunks = pairhist_geom<8, true>(L, nseq).nchunks; break;
        case 4: nchunks = pairhist_geom<4, true>(L, nseq).nchunks; break;
        default: break;
    }
    return 256 + usite_bytes(L, q) + (size_t)std::max<uint32_t>(nchunks, 1) * npairs_of(L) * q * q * 4;
}

extern "C" int mi3_weighted_marg(const float *weights, const uint32_t *seqmem, uint32_t buflen,
                                 uint32_t nseq, float *bimarg, uint32_t L, uint32_t q, const uint8_t *cons,
                                 void *workspace, size_t ws_bytes, void *stream) {
    if (!weights || !seqmem || !bimarg || !workspace) return fail(MI3_ERR_ARG, "mi3_weighted_marg: null pointer");
    if (L < 2 || q < 1 || q > 255 || nseq > buflen)
        return fail(MI3_ERR_ARG, "mi3_weighted_marg: bad L/q/nseq");
    if (nseq == 0) {
        cudaMemsetAsync(bimarg, 0, (size_t)npairs_of(L) * q * q * 4, as_stream(stream));
        return check_launch("mi3_weighted_marg: memset");
    }
    if (ws_bytes < mi3_weighted_marg_workspace(L, q, nseq))
        return fail(MI3_ERR_WORKSPACE, "mi3_weighted_marg: workspace too small");
    if (!aligned(workspace, 256)) return fail(MI3_ERR_ALIGN, "mi3_weighted_marg: workspace must be 256B aligned");
    return dispatch_pairhist<true>(seqmem, buflen, nseq, weights, reinterpret_cast<unsigned char *>(workspace),
                                   bimarg, L, q, cons, as_stream(stream));
}

extern "C" size_t mi3_site_consensus_workspace(uint32_t L, uint32_t q) { return (size_t)L * q * 8; }

extern "C" int mi3_site_consensus(const uint32_t *seqmem, uint32_t buflen, uint32_t nseq, uint32_t L, uint32_t q,
                                  uint8_t *cons, void *workspace, size_t ws_bytes, void *stream) {
    if (!seqmem || !cons || !workspace) return fail(MI3_ERR_ARG, "mi3_site_consensus: null pointer");
    if (L < 1 || q < 1 || q > 255 || nseq > buflen) return fail(MI3_ERR_ARG, "mi3_site_consensus: bad L/q/nseq");
    if ((size_t)L * q * 4 + L > 160 * 1024) return fail(MI3_ERR_ARG, "mi3_site_consensus: L*q too large");
    if (ws_bytes < mi3_site_consensus_workspace(L, q))
        return fail(MI3_ERR_WORKSPACE, "mi3_site_consensus: workspace too small");
    if (!aligned(workspace, 8)) return fail(MI3_ERR_ALIGN, "mi3_site_consensus: workspace alignment");
    cudaStream_t st = as_stream(stream);
    auto *cnt = reinterpret_cast<unsigned long long *>(workspace);
    if (cudaMemsetAsync(cnt, 0, (size_t)L * q * 8, st) != cudaSuccess)
        return check_launch("mi3_site_consensus: memset");
    if (nseq > 0) {
        const uint32_t per_cta = std::max<uint32_t>(256, (nseq + 148 * 4 - 1) / (148 * 4));
        const size_t ssm = (size_t)L * q * 4 + L;
        if (ssm > 48 * 1024)
            cudaFuncSetAttribute(k_site_hist<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ssm);
        k_site_hist<false, false><<<(nseq + per_cta - 1) / per_cta, 256, ssm, st>>>(
            seqmem, buflen, nseq, nullptr, nullptr, 0, nullptr, cnt, nullptr, L, q, per_cta);
        int rc = check_launch("mi3_site_consensus: counts");
        if (rc) return rc;
    }
    k_argmax_sites<<<(L + 127) / 128, 128, 0, st>>>(cnt, cons, L, q);
    return check_launch("mi3_site_consensus: argmax");
}

extern "C" int mi3_bicounts_to_bimarg(const uint32_t *bicount, float *bimarg, uint32_t nseq, uint32_t L,
                                      uint32_t q, void *stream) {
    if (!bicount || !bimarg) return fail(MI3_ERR_ARG, "mi3_bicounts_to_bimarg: null pointer");
    if (L < 2 || q < 1) return fail(MI3_ERR_ARG, "mi3_bicounts_to_bimarg: bad L/q");
    uint64_t n = npairs_of(L) * q * q;
    k_bicounts_to_bimarg<<<(uint32_t)((n + 255) / 256), 256, 0, as_stream(stream)>>>(bicount, bimarg,
                                                                                    (float)nseq, n);
    return check_launch("mi3_bicounts_to_bimarg");
}

extern "C" int mi3_renormalize_bimarg(float *bimarg, uint32_t L, uint32_t q, void *stream) {
    if (!bimarg) return fail(MI3_ERR_ARG, "mi3_renormalize_bimarg: null pointer");
    if (L < 2 || q < 1 || q * q > 4096) return fail(MI3_ERR_ARG, "mi3_renormalize_bimarg: bad L/q");
    uint64_t np = npairs_of(L);
    uint32_t qq = q * q;
    uint32_t tb = 256;
    size_t smem = (size_t)(tb / 32) * qq * 4;
    uint32_t grid = (uint32_t)std::min<uint64_t>((np + 7) / 8, 148 * 16);
    k_renormalize<<<grid, tb, smem, as_stream(stream)>>>(bimarg, np, qq);
    return check_launch("mi3_renormalize_bimarg");
}

extern "C" int mi3_repack_seqs_T(const uint32_t *seq4, uint32_t buf4len, uint32_t *seqL, uint32_t buf1len,
                                 uint32_t L, void *stream) {
    if (!seq4 || !seqL) return fail(MI3_ERR_ARG, "mi3_repack_seqs_T: null pointer");
    if (L < 1 || buf1len == 0) return fail(MI3_ERR_ARG, "mi3_repack_seqs_T: bad sizes");
    dim3 grid((buf1len + 255) / 256, L);
    k_repack_T<<<grid, 256, 0, as_stream(stream)>>>(seq4, buf4len, seqL, buf1len, L);
    return check_launch("mi3_repack_seqs_T");
}
