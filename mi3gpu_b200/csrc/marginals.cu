// marginals.cu -- pair histograms of the walkers' sequences.
//
//   mi3_bicounts        exact uint32 counts (countBivariate, mcmc.cl:462-516)
//   mi3_weighted_marg   float weighted sums (weightedMarg, mcmc.cl:646-718)
//   mi3_bicounts_to_bimarg, mi3_renormalize_bimarg, mi3_repack_seqs_T
//
// The histogram kernels use the slice tiling of tiling.cuh: a CTA keeps the
// B*B pair histograms (q*q bins each) of one block pair in shared memory,
// increments them with shared-memory atomics for a chunk of sequences, and
// flushes them once.  Counts are integers, so they are exact whatever the
// order.
#include "tiling.cuh"

namespace mi3 {

template <int B, typename T>
__device__ __forceinline__ void hist_flush(const T *h, T *out, uint32_t L, uint32_t q,
                                           uint32_t i0, uint32_t j0, bool accumulate) {
    const uint32_t qq = q * q;
    for (int ii = 0; ii < B; ++ii) {
        uint32_t i = i0 + ii;
        if (i + 1 >= L) break;
        uint32_t jlo = max(j0, i + 1), jhi = min(j0 + B, L);
        if (jlo >= jhi) continue;
        T *dst = out + pair_index(i, jlo, L) * qq;
        const T *src = h + ((size_t)ii * B + (jlo - j0)) * qq;
        uint32_t cnt = (jhi - jlo) * qq;
        for (uint32_t k = threadIdx.x; k < cnt; k += blockDim.x) {
            T v = src[k];
            if (accumulate) {
                if (v != T(0)) atomicAdd(&dst[k], v);
            } else {
                dst[k] = v;
            }
        }
    }
}

// WEIGHTED=false: uint32 counts.  WEIGHTED=true: float sums of weights[n].
template <int B, bool WEIGHTED>
__global__ void __launch_bounds__(512) k_pairhist(const uint32_t *__restrict__ seq, uint32_t buflen,
                                                  uint32_t nseq, const float *__restrict__ weights,
                                                  void *out, uint32_t L, uint32_t q, SliceGeom g) {
    using T = typename std::conditional<WEIGHTED, float, uint32_t>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *h = reinterpret_cast<T *>(smem_raw);  // [B*B][q*q]
    const uint32_t qq = q * q;
    const uint32_t s = blockIdx.x % g.nslices;
    const uint32_t chunk = blockIdx.x / g.nslices;
    uint32_t bi, bj;
    slice_coords(s, g.nb, bi, bj);
    const uint32_t i0 = bi * B, j0 = bj * B;
    const uint32_t nh = B * B * qq;
    for (uint32_t k = threadIdx.x; k < nh; k += blockDim.x) h[k] = T(0);
    __syncthreads();

    const uint32_t swords = (L - 1) / 4 + 1;
    const uint32_t nbeg = chunk * g.chunk;
    const uint32_t nend = min(nseq, nbeg + g.chunk);
    for (uint32_t n = nbeg + threadIdx.x; n < nend; n += blockDim.x) {
        uint32_t wI[B / 4], wJ[B / 4];
        load_block_words<B>(seq, buflen, n, bi, swords, wI);
        load_block_words<B>(seq, buflen, n, bj, swords, wJ);
        T inc;
        if constexpr (WEIGHTED) inc = __ldg(&weights[n]);
        else inc = 1u;
#pragma unroll
        for (int ii = 0; ii < B; ++ii) {
            uint32_t i = i0 + ii;
            if (i >= L) break;
            T *row = h + (size_t)ii * B * qq + block_byte<B>(wI, ii, q - 1) * q;
#pragma unroll
            for (int jj = 0; jj < B; ++jj) {
                uint32_t j = j0 + jj;
                if (j < L && j > i) atomicAdd(&row[(size_t)jj * qq + block_byte<B>(wJ, jj, q - 1)], inc);
            }
        }
    }
    __syncthreads();
    hist_flush<B, T>(h, reinterpret_cast<T *>(out), L, q, i0, j0, g.nchunks > 1);
}

template <int B, bool WEIGHTED>
static int launch_pairhist(const uint32_t *seq, uint32_t buflen, uint32_t nseq, const float *w,
                           void *out, uint32_t L, uint32_t q, cudaStream_t st, bool split) {
    SliceGeom g = make_geom(L, B, nseq, split ? 148 * 8 : 1, split ? 2048 : nseq);
    size_t smem = (size_t)B * B * q * q * 4;
    cudaFuncSetAttribute(k_pairhist<B, WEIGHTED>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    uint64_t nblk = (uint64_t)g.nslices * g.nchunks;
    if (nblk > 0x7fffffffull) return fail(MI3_ERR_ARG, "pair histogram: grid too large");
    if (g.nchunks > 1) {
        size_t bytes = (size_t)npairs_of(L) * q * q * 4;
        if (cudaMemsetAsync(out, 0, bytes, st) != cudaSuccess) return check_launch("pair histogram: memset");
    }
    k_pairhist<B, WEIGHTED><<<(uint32_t)nblk, 512, smem, st>>>(seq, buflen, nseq, w, out, L, q, g);
    return check_launch(WEIGHTED ? "mi3_weighted_marg" : "mi3_bicounts");
}

template <bool WEIGHTED>
static int dispatch_pairhist(const uint32_t *seq, uint32_t buflen, uint32_t nseq, const float *w,
                             void *out, uint32_t L, uint32_t q, cudaStream_t st, bool split) {
    switch (pick_block(q, 116 * 1024)) {
        case 32: return launch_pairhist<32, WEIGHTED>(seq, buflen, nseq, w, out, L, q, st, split);
        case 16: return launch_pairhist<16, WEIGHTED>(seq, buflen, nseq, w, out, L, q, st, split);
        case 8: return launch_pairhist<8, WEIGHTED>(seq, buflen, nseq, w, out, L, q, st, split);
        case 4: return launch_pairhist<4, WEIGHTED>(seq, buflen, nseq, w, out, L, q, st, split);
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
    return dispatch_pairhist<false>(seqmem, buflen, nseq, nullptr, bicount, L, q, as_stream(stream), true);
}

extern "C" int mi3_weighted_marg(const float *weights, const uint32_t *seqmem, uint32_t buflen,
                                 uint32_t nseq, float *bimarg, uint32_t L, uint32_t q, void *stream) {
    if (!weights || !seqmem || !bimarg) return fail(MI3_ERR_ARG, "mi3_weighted_marg: null pointer");
    if (L < 2 || q < 1 || q > 255 || nseq > buflen)
        return fail(MI3_ERR_ARG, "mi3_weighted_marg: bad L/q/nseq");
    if (nseq == 0) {
        cudaMemsetAsync(bimarg, 0, (size_t)npairs_of(L) * q * q * 4, as_stream(stream));
        return check_launch("mi3_weighted_marg: memset");
    }
    return dispatch_pairhist<true>(seqmem, buflen, nseq, weights, bimarg, L, q, as_stream(stream), false);
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
