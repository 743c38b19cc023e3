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
__device__ __forceinline__ int fixed_shift(float wmax, uint32_t chunk) {
    if (!(wmax > 0.0f)) return 40;
    double lim = 4294967295.0 / ((double)chunk * (double)wmax);
    int s = (int)floor(log2(lim));
    return min(s, 40);
}

template <int B, bool WEIGHTED>
__global__ void __launch_bounds__(512) k_pairhist(const uint32_t *__restrict__ seq, uint32_t buflen,
                                                  uint32_t nseq, const float *__restrict__ weights,
                                                  const unsigned int *__restrict__ wmax_bits, void *out,
                                                  uint32_t L, uint32_t q, SliceGeom g) {
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
    __syncthreads();

    const uint32_t swords = (L - 1) / 4 + 1;
    const uint32_t nbeg = chunk * g.chunk;
    const uint32_t nend = min(nseq, nbeg + g.chunk);
    const uint32_t stride = 2 * blockDim.x;
    for (uint32_t n = nbeg + threadIdx.x; n < nend; n += stride) {
        const uint32_t n2 = n + blockDim.x;
        const bool two = n2 < nend;
        uint32_t wI[B / 4], wJ[B / 4], vI[B / 4], vJ[B / 4];
        load_block_words<B>(seq, buflen, n, bi, swords, wI);
        load_block_words<B>(seq, buflen, n, bj, swords, wJ);
        load_block_words<B>(seq, buflen, two ? n2 : n, bi, swords, vI);
        load_block_words<B>(seq, buflen, two ? n2 : n, bj, swords, vJ);
        uint32_t inc1 = 1u, inc2 = two ? 1u : 0u;
        if constexpr (WEIGHTED) {
            inc1 = __float2uint_rn(__ldg(&weights[n]) * scale);
            inc2 = two ? __float2uint_rn(__ldg(&weights[n2]) * scale) : 0u;
        }
#pragma unroll
        for (int ii = 0; ii < B; ++ii) {
            uint32_t i = i0 + ii;
            if (i >= L) break;
            uint32_t *row1 = h + (size_t)ii * B * qq + block_byte<B>(wI, ii, q - 1) * q;
            uint32_t *row2 = h + (size_t)ii * B * qq + block_byte<B>(vI, ii, q - 1) * q;
#pragma unroll
            for (int jj = 0; jj < B; ++jj) {
                uint32_t j = j0 + jj;
                if (j < L && j > i) {
                    atomicAdd(&row1[(size_t)jj * qq + block_byte<B>(wJ, jj, q - 1)], inc1);
                    if (two) atomicAdd(&row2[(size_t)jj * qq + block_byte<B>(vJ, jj, q - 1)], inc2);
                }
            }
        }
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
                if (v) atomicAdd(reinterpret_cast<unsigned long long *>(out) + dst0 + k, (unsigned long long)v);
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

// Fixed-point accumulators -> float weighted bimarginals.
__global__ void k_fixed_to_float(const unsigned long long *__restrict__ acc, const unsigned int *wmax_bits,
                                 uint32_t chunk, float *out, uint64_t n) {
    uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int s = fixed_shift(__uint_as_float(*wmax_bits), chunk);
    out[k] = (float)ldexp((double)acc[k], -s);
}

constexpr uint32_t WMARG_CHUNK = 65536;  // sequences per CTA (fixed-point headroom)

template <int B, bool WEIGHTED>
static int launch_pairhist(const uint32_t *seq, uint32_t buflen, uint32_t nseq, const float *w,
                           unsigned char *ws, void *out, uint32_t L, uint32_t q, cudaStream_t st) {
    SliceGeom g = make_geom(L, B, nseq, 148 * 8, 2048);
    if (WEIGHTED && g.chunk > WMARG_CHUNK) {
        g.chunk = WMARG_CHUNK;
        g.nchunks = (nseq + g.chunk - 1) / g.chunk;
    }
    size_t smem = (size_t)B * B * q * q * 4;
    cudaFuncSetAttribute(k_pairhist<B, WEIGHTED>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    uint64_t nblk = (uint64_t)g.nslices * g.nchunks;
    if (nblk > 0x7fffffffull) return fail(MI3_ERR_ARG, "pair histogram: grid too large");
    const uint64_t nbins = npairs_of(L) * q * q;
    unsigned int *wmax = nullptr;
    void *dst = out;
    if (WEIGHTED) {
        wmax = reinterpret_cast<unsigned int *>(ws);
        dst = ws + 256;
        if (cudaMemsetAsync(ws, 0, 256 + nbins * 8, st) != cudaSuccess) return check_launch("weighted marg: memset");
        k_wmax<<<296, 512, 0, st>>>(w, nseq, wmax);
    } else if (g.nchunks > 1) {
        if (cudaMemsetAsync(out, 0, nbins * 4, st) != cudaSuccess) return check_launch("bicounts: memset");
    }
    k_pairhist<B, WEIGHTED><<<(uint32_t)nblk, 512, smem, st>>>(seq, buflen, nseq, w, wmax, dst, L, q, g);
    if (WEIGHTED)
        k_fixed_to_float<<<(uint32_t)((nbins + 255) / 256), 256, 0, st>>>(
            reinterpret_cast<const unsigned long long *>(dst), wmax, g.chunk, reinterpret_cast<float *>(out), nbins);
    return check_launch(WEIGHTED ? "mi3_weighted_marg" : "mi3_bicounts");
}

template <bool WEIGHTED>
static int dispatch_pairhist(const uint32_t *seq, uint32_t buflen, uint32_t nseq, const float *w,
                             unsigned char *ws, void *out, uint32_t L, uint32_t q, cudaStream_t st) {
    switch (pick_block(q, 116 * 1024)) {
        case 32: return launch_pairhist<32, WEIGHTED>(seq, buflen, nseq, w, ws, out, L, q, st);
        case 16: return launch_pairhist<16, WEIGHTED>(seq, buflen, nseq, w, ws, out, L, q, st);
        case 8: return launch_pairhist<8, WEIGHTED>(seq, buflen, nseq, w, ws, out, L, q, st);
        case 4: return launch_pairhist<4, WEIGHTED>(seq, buflen, nseq, w, ws, out, L, q, st);
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
    return dispatch_pairhist<false>(seqmem, buflen, nseq, nullptr, nullptr, bicount, L, q, as_stream(stream));
}

extern "C" size_t mi3_weighted_marg_workspace(uint32_t L, uint32_t q) {
    return 256 + (size_t)npairs_of(L) * q * q * 8;
}

extern "C" int mi3_weighted_marg(const float *weights, const uint32_t *seqmem, uint32_t buflen,
                                 uint32_t nseq, float *bimarg, uint32_t L, uint32_t q, void *workspace,
                                 size_t ws_bytes, void *stream) {
    if (!weights || !seqmem || !bimarg || !workspace) return fail(MI3_ERR_ARG, "mi3_weighted_marg: null pointer");
    if (L < 2 || q < 1 || q > 255 || nseq > buflen)
        return fail(MI3_ERR_ARG, "mi3_weighted_marg: bad L/q/nseq");
    if (nseq == 0) {
        cudaMemsetAsync(bimarg, 0, (size_t)npairs_of(L) * q * q * 4, as_stream(stream));
        return check_launch("mi3_weighted_marg: memset");
    }
    if (ws_bytes < mi3_weighted_marg_workspace(L, q))
        return fail(MI3_ERR_WORKSPACE, "mi3_weighted_marg: workspace too small");
    if (!aligned(workspace, 256)) return fail(MI3_ERR_ALIGN, "mi3_weighted_marg: workspace must be 256B aligned");
    return dispatch_pairhist<true>(seqmem, buflen, nseq, weights, reinterpret_cast<unsigned char *>(workspace),
                                   bimarg, L, q, as_stream(stream));
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
