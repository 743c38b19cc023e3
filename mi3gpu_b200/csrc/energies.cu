// energies.cu -- Potts energies E(s) = sum_{i<j} J_ij(s_i, s_j).
//
// Slice-tiled (tiling.cuh): a CTA holds the couplings of one block pair in
// shared memory and streams a chunk of sequences through it; each thread
// sums its sequence's gathered couplings (float within a site row of at most
// B terms, double across rows) and adds the slice total to a per-sequence
// 64-bit fixed-point accumulator (scale 2^40) with an integer atomic.
// Integer addition is associative, so the result does not depend on CTA
// order: energies are deterministic.  The float row sums bound the error at
// about B*2^-24 of the largest row sum per row, far below the final
// rounding to float for the energies the sampler meets.  The reference sums each
// sequence serially with Kahan compensation in float (getEnergiesf,
// mcmc.cl:249-336); this result is at least as accurate.
#include <mutex>

#include "tiling.cuh"

namespace mi3 {

constexpr double FIX_SCALE = 1099511627776.0;  // 2^40
constexpr double FIX_INV = 1.0 / 1099511627776.0;

// Energy of one sequence over the pairs of one slice: each site row of B
// couplings is summed in float (at most B terms) and the row sums in double.
// CONS: the table is in the consensus gauge (tiling.cuh), so pairs where
// either residue is its site's consensus contribute zero and are skipped.
template <int B, int K, bool CONS>
__device__ __forceinline__ double slice_energy(const float *js, const uint32_t (&wI)[B / 4],
                                               const uint32_t (&wJ)[B / 4], const uint32_t (&cI)[B / 4],
                                               const uint32_t (&cJ)[B / 4], uint32_t q, uint32_t qq,
                                               uint32_t i0, uint32_t j0, uint32_t L) {
    uint32_t col[B];
    slice_cols<B>(wJ, q, qq, col);
    double e = 0.0;
    if constexpr (!CONS) {
#pragma unroll
        for (int ii = 0; ii < B; ++ii) {
            if (K == SLICE_EDGE && i0 + ii >= L) break;
            const uint32_t row = slice_row<B>(wI, ii, q, qq);
            float r = 0.0f;
#pragma unroll
            for (int jj = 0; jj < B; ++jj)
                if (slice_pair_valid<K>(ii, jj, i0, j0, L)) r += js[row + col[jj]];
            e += (double)r;
        }
    } else {
        uint32_t mI[B / 4], mJ[B / 4];
        cons_masks<B>(wI, cI, mI);
        cons_masks<B>(wJ, cJ, mJ);
        const uint32_t cb = cons_bits<B>(mJ);
        const uint32_t base = (uint32_t)__cvta_generic_to_shared(js);
#pragma unroll
        for (int ii = 0; ii < B; ++ii) {
            if (K == SLICE_EDGE && i0 + ii >= L) break;
            const uint32_t row = slice_row<B>(wI, ii, q, qq);
            const uint32_t rb = cons_off<B>(mI, ii) ? cb : 0u;  // active columns of this row
            float v[B];
#pragma unroll
            for (int jj = 0; jj < B; ++jj)
                v[jj] = slice_pair_valid<K>(ii, jj, i0, j0, L) ? lds_if(base + 4u * (row + col[jj]), rb & (1u << jj))
                                                               : 0.0f;
            float r = 0.0f;
#pragma unroll
            for (int jj = 0; jj < B; ++jj) r += v[jj];
            e += (double)r;
        }
    }
    return e;
}

template <int B, int K, bool CONS>
__device__ __forceinline__ void energies_chunk(const float *js, const uint32_t *__restrict__ seq, uint32_t buflen,
                                               uint32_t nbeg, uint32_t nend, unsigned long long *acc,
                                               uint32_t L, uint32_t q, uint32_t bi, uint32_t bj,
                                               const uint32_t (&cI)[B / 4], const uint32_t (&cJ)[B / 4]) {
    const uint32_t qq = q * q, swords = (L - 1) / 4 + 1;
    const uint32_t i0 = bi * B, j0 = bj * B;
    if constexpr (B <= 8 || !CONS) {
        // two sequences per thread: two independent gather/add chains in flight
        for (uint32_t n = nbeg + threadIdx.x; n < nend; n += 2 * blockDim.x) {
            const uint32_t n2 = n + blockDim.x;
            const bool two = n2 < nend;
            uint32_t wI[B / 4], wJ[B / 4], vI[B / 4], vJ[B / 4];
            load_block_words<B>(seq, buflen, n, bi, swords, wI);
            load_block_words<B>(seq, buflen, n, bj, swords, wJ);
            load_block_words<B>(seq, buflen, two ? n2 : n, bi, swords, vI);
            load_block_words<B>(seq, buflen, two ? n2 : n, bj, swords, vJ);
            const double e1 = slice_energy<B, K, CONS>(js, wI, wJ, cI, cJ, q, qq, i0, j0, L);
            const double e2 = slice_energy<B, K, CONS>(js, vI, vJ, cI, cJ, q, qq, i0, j0, L);
            atomicAdd(&acc[n], (unsigned long long)__double2ll_rn(e1 * FIX_SCALE));
            if (two) atomicAdd(&acc[n2], (unsigned long long)__double2ll_rn(e2 * FIX_SCALE));
        }
    } else {
        // 16-site blocks with consensus masks: one sequence per thread keeps
        // the offsets and masks in registers
        for (uint32_t n = nbeg + threadIdx.x; n < nend; n += blockDim.x) {
            uint32_t wI[B / 4], wJ[B / 4];
            load_block_words<B>(seq, buflen, n, bi, swords, wI);
            load_block_words<B>(seq, buflen, n, bj, swords, wJ);
            const double e1 = slice_energy<B, K, CONS>(js, wI, wJ, cI, cJ, q, qq, i0, j0, L);
            atomicAdd(&acc[n], (unsigned long long)__double2ll_rn(e1 * FIX_SCALE));
        }
    }
}

// Full slices with lanes over pairs (tiling.cuh): the table is [cell][P];
// lane w visits pair (t + w) mod P at step t.  Each sequence's B*B terms are
// summed as B float partial sums (step rows th, at most B terms each) added
// in double, then in fixed point as above.
template <int B>
__device__ __forceinline__ double lane_energy(uint32_t jbase, const uint32_t (&row)[B], const uint32_t (&col)[B],
                                              uint32_t wl) {
    float part[B];
#pragma unroll
    for (int th = 0; th < B; ++th) part[th] = 0.0f;
#pragma unroll
    for (int tl = 0; tl < B; ++tl) {
        const bool carry = tl + wl >= (uint32_t)B;
        const uint32_t c = jbase + col[tl];
#pragma unroll
        for (int th = 0; th < B; ++th) {
            const uint32_t r = carry ? row[(th + 1) & (B - 1)] : row[th];
            float v;
            asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(c + r));
            part[th] += v;
        }
    }
    double e = 0.0;
#pragma unroll
    for (int th = 0; th < B; ++th) e += (double)part[th];
    return e;
}

template <int B>
__device__ __forceinline__ void energies_chunk_lanes(const float *js, const uint32_t *__restrict__ seq, uint32_t buflen,
                                                     uint32_t nbeg, uint32_t nend, unsigned long long *acc,
                                                     uint32_t L, uint32_t q, uint32_t bi, uint32_t bj) {
    const uint32_t swords = (L - 1) / 4 + 1;
    const uint32_t lane = threadIdx.x & 31, wl = lane % B;
    const uint32_t jbase = (uint32_t)__cvta_generic_to_shared(js);
    if constexpr (B == 16) {
        // 256 terms per sequence: one sequence per thread has loads enough
        // in flight (16 independent partial sums) and fits the registers
        for (uint32_t n = nbeg + threadIdx.x; n < nend; n += blockDim.x) {
            uint32_t wI[B / 4], wJ[B / 4];
            load_block_words<B>(seq, buflen, n, bi, swords, wI);
            load_block_words<B>(seq, buflen, n, bj, swords, wJ);
            uint32_t row[B], col[B];
            lane_offsets<B>(wI, wJ, q, lane, row, col);
            const double e1 = lane_energy<B>(jbase, row, col, wl);
            atomicAdd(&acc[n], (unsigned long long)__double2ll_rn(e1 * FIX_SCALE));
        }
        return;
    }
    // two sequences per thread: two independent chains of loads in flight
    for (uint32_t n = nbeg + threadIdx.x; n < nend; n += 2 * blockDim.x) {
        const uint32_t n2 = n + blockDim.x;
        const bool two = n2 < nend;
        uint32_t wI[B / 4], wJ[B / 4], vI[B / 4], vJ[B / 4];
        load_block_words<B>(seq, buflen, n, bi, swords, wI);
        load_block_words<B>(seq, buflen, n, bj, swords, wJ);
        load_block_words<B>(seq, buflen, two ? n2 : n, bi, swords, vI);
        load_block_words<B>(seq, buflen, two ? n2 : n, bj, swords, vJ);
        uint32_t row[B], col[B];
        lane_offsets<B>(wI, wJ, q, lane, row, col);
        const double e1 = lane_energy<B>(jbase, row, col, wl);
        lane_offsets<B>(vI, vJ, q, lane, row, col);
        const double e2 = lane_energy<B>(jbase, row, col, wl);
        atomicAdd(&acc[n], (unsigned long long)__double2ll_rn(e1 * FIX_SCALE));
        if (two) atomicAdd(&acc[n2], (unsigned long long)__double2ll_rn(e2 * FIX_SCALE));
    }
}

template <int B, bool CONS>
__global__ void __launch_bounds__(512, 2) k_energies(const float *__restrict__ J,
                                                     const uint32_t *__restrict__ seq, uint32_t buflen,
                                                     uint32_t nseq, unsigned long long *acc, uint32_t L,
                                                     uint32_t q, SliceGeom g, const uint8_t *__restrict__ cons) {
    extern __shared__ __align__(16) float js[];  // [B*B][q*q]
    const uint32_t qq = q * q;
    const uint32_t s = blockIdx.x % g.nslices;
    const uint32_t chunk = blockIdx.x / g.nslices;
    uint32_t bi, bj;
    slice_coords(s, g.nb, bi, bj);
    const uint32_t i0 = bi * B, j0 = bj * B;
    const int kind = slice_kind(bi, bj, j0, B, L);
    const uint32_t nbeg = chunk * g.chunk;
    const uint32_t nend = min(nseq, nbeg + g.chunk);

    if constexpr (!CONS && B >= 8) {
        if (kind == SLICE_FULL) {
            // cell-major table [cell][P] for lanes over pairs: lane l
            // stages cell c0 + l % 8 of pair p0 + l / 8 (global reads of 8
            // consecutive cells of 4 pairs)
            constexpr uint32_t P = B * B;
            const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
            const uint32_t cgroups = (qq + 7) / 8;
            for (uint32_t t = warp; t < cgroups * (P / 4); t += nwarps) {
                const uint32_t c = (t % cgroups) * 8 + (lane & 7), p = (t / cgroups) * 4 + (lane >> 3);
                if (c < qq) js[c * P + p] = __ldg(&J[pair_index(i0 + p / B, j0 + p % B, L) * qq + c]);
            }
            __syncthreads();
            energies_chunk_lanes<B>(js, seq, buflen, nbeg, nend, acc, L, q, bi, bj);
            return;
        }
    }

    // Stage the slice's couplings: for each i, pairs (i, jlo..jhi-1) are
    // contiguous in the packed table.
    for (int ii = 0; ii < B; ++ii) {
        uint32_t i = i0 + ii;
        if (i + 1 >= L) break;
        uint32_t jlo = max(j0, i + 1), jhi = min(j0 + B, L);
        if (jlo >= jhi) continue;
        const float *src = J + pair_index(i, jlo, L) * qq;
        float *dst = js + ((size_t)ii * B + (jlo - j0)) * qq;
        uint32_t cnt = (jhi - jlo) * qq;
        for (uint32_t k = threadIdx.x; k < cnt; k += blockDim.x) dst[k] = __ldg(&src[k]);
    }
    uint32_t cI[B / 4] = {}, cJ[B / 4] = {};
    if constexpr (CONS) {
        load_cons_words<B>(cons, bi, L, cI);
        load_cons_words<B>(cons, bj, L, cJ);
    }
    __syncthreads();

    switch (kind) {
        case SLICE_FULL:
            energies_chunk<B, SLICE_FULL, CONS>(js, seq, buflen, nbeg, nend, acc, L, q, bi, bj, cI, cJ);
            break;
        case SLICE_DIAG:
            energies_chunk<B, SLICE_DIAG, CONS>(js, seq, buflen, nbeg, nend, acc, L, q, bi, bj, cI, cJ);
            break;
        default:
            energies_chunk<B, SLICE_EDGE, CONS>(js, seq, buflen, nbeg, nend, acc, L, q, bi, bj, cI, cJ);
            break;
    }
}

__global__ void k_energies_final(const unsigned long long *__restrict__ acc, float *E, uint32_t n) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) E[k] = (float)((double)(long long)acc[k] * FIX_INV);
}

template <int B, bool CONS>
static int launch_energies(const float *J, const uint32_t *seq, uint32_t buflen, uint32_t nseq,
                           unsigned long long *acc, uint32_t L, uint32_t q, const uint8_t *cons, cudaStream_t st) {
    SliceGeom g = make_geom(L, B, nseq, 148 * 8, 2048);
    size_t smem = (size_t)B * B * q * q * 4;
    cudaFuncSetAttribute(k_energies<B, CONS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    uint64_t nblk = (uint64_t)g.nslices * g.nchunks;
    if (nblk > 0x7fffffffull) return fail(MI3_ERR_ARG, "mi3_energies: grid too large");
    k_energies<B, CONS><<<(uint32_t)nblk, 512, smem, st>>>(J, seq, buflen, nseq, acc, L, q, g, cons);
    return check_launch("mi3_energies");
}

template <bool CONS>
static int dispatch_energies(const float *J, const uint32_t *seq, uint32_t buflen, uint32_t nseq,
                             unsigned long long *acc, uint32_t L, uint32_t q, const uint8_t *cons,
                             cudaStream_t st) {
    switch (pick_block(q, 116 * 1024, 16)) {
        case 16: return launch_energies<16, CONS>(J, seq, buflen, nseq, acc, L, q, cons, st);
        case 8: return launch_energies<8, CONS>(J, seq, buflen, nseq, acc, L, q, cons, st);
        case 4: return launch_energies<4, CONS>(J, seq, buflen, nseq, acc, L, q, cons, st);
        default: return fail(MI3_ERR_ARG, "mi3_energies: q too large");
    }
}

// ------------------------------------------------------- consensus gauge
// J'(a,b) = J(a,b) - J(a,c_j) - J(c_i,b) + J(c_i,c_j), computed in double and
// rounded once; row c_i and column c_j of J' are exactly zero.  The removed
// parts: x_i(a) = J(a,c_j) - J(c_i,c_j) for site i, y_j(b) = J(c_i,b) -
// J(c_i,c_j) for site j, and the constant J(c_i,c_j), so that
// J(a,b) = J'(a,b) + x_i(a) + y_j(b) + J(c_i,c_j).
__global__ void k_cons_gauge(const float *__restrict__ J, const uint8_t *__restrict__ cons, float *Jc,
                             uint32_t L, uint32_t q) {
    const uint32_t p = blockIdx.x;
    __shared__ uint32_t ij[2];
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
    __syncthreads();
    const uint32_t qq = q * q;
    const uint32_t ci = min((uint32_t)cons[ij[0]], q - 1), cj = min((uint32_t)cons[ij[1]], q - 1);
    const float *Jp = J + (size_t)p * qq;
    const double cc = Jp[ci * q + cj];
    for (uint32_t e = threadIdx.x; e < qq; e += blockDim.x) {
        const uint32_t a = e / q, b = e - a * q;
        const double v = ((double)Jp[e] - (double)Jp[a * q + cj]) - ((double)Jp[ci * q + b] - cc);
        Jc[(size_t)p * qq + e] = (float)v;
    }
}

// Site fields of the consensus gauge, h[k][a] = sum over the pairs of site k
// of its x or y part, and the per-site share of the constant (pairs (k, j>k)).
__global__ void k_cons_fields(const float *__restrict__ J, const uint8_t *__restrict__ cons, double *h,
                              double *cpart, uint32_t L, uint32_t q) {
    const uint32_t k = blockIdx.x, qq = q * q;
    const uint32_t ck = min((uint32_t)cons[k], q - 1);
    for (uint32_t a = threadIdx.x; a < q; a += blockDim.x) {
        double acc = 0.0;
        for (uint32_t i = 0; i < k; ++i) {  // pair (i, k): site k is the column
            const float *Jp = J + pair_index(i, k, L) * qq;
            const uint32_t ci = min((uint32_t)cons[i], q - 1);
            acc += (double)Jp[ci * q + a] - (double)Jp[ci * q + ck];
        }
        for (uint32_t j = k + 1; j < L; ++j) {  // pair (k, j): site k is the row
            const float *Jp = J + pair_index(k, j, L) * qq;
            const uint32_t cj = min((uint32_t)cons[j], q - 1);
            acc += (double)Jp[a * q + cj] - (double)Jp[ck * q + cj];
        }
        h[(size_t)k * q + a] = acc;
    }
    if (threadIdx.x == 0) {
        double c = 0.0;
        for (uint32_t j = k + 1; j < L; ++j)
            c += (double)J[pair_index(k, j, L) * qq + ck * q + min((uint32_t)cons[j], q - 1)];
        cpart[k] = c;
    }
}

// E[n] = pair sums (fixed point) + sum_i h[i][s_i] + constant.
__global__ void __launch_bounds__(256) k_energies_final_cons(const unsigned long long *__restrict__ acc,
                                                             const uint32_t *__restrict__ seq, uint32_t buflen,
                                                             const double *__restrict__ h,
                                                             const double *__restrict__ cpart, float *E,
                                                             uint32_t n, uint32_t L, uint32_t q) {
    extern __shared__ double hs[];  // [L*q] fields, then the constant
    for (uint32_t k = threadIdx.x; k < L * q; k += blockDim.x) hs[k] = h[k];
    if (threadIdx.x == 0) {
        double c = 0.0;
        for (uint32_t k = 0; k < L; ++k) c += cpart[k];
        hs[L * q] = c;
    }
    __syncthreads();
    const uint32_t swords = (L - 1) / 4 + 1;
    for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += gridDim.x * blockDim.x) {
        double e = (double)(long long)acc[m] * FIX_INV;
        double f = 0.0;
        for (uint32_t w = 0; w < swords; ++w) {
            const uint32_t word = __ldg(&seq[(size_t)w * buflen + m]);
#pragma unroll
            for (uint32_t t = 0; t < 4; ++t) {
                const uint32_t site = 4 * w + t;
                if (site < L) f += hs[site * q + min((word >> (8 * t)) & 0xffu, q - 1)];
            }
        }
        E[m] = (float)(e + f + hs[L * q]);
    }
}

}  // namespace mi3

using namespace mi3;

extern "C" size_t mi3_energies_workspace(uint32_t nseq) { return (size_t)nseq * 8; }

extern "C" int mi3_energies(const float *J, const uint32_t *seqmem, uint32_t buflen, uint32_t nseq,
                            float *energies, uint32_t L, uint32_t q, void *workspace,
                            size_t ws_bytes, void *stream) {
    if (!J || !seqmem || !energies || !workspace)
        return fail(MI3_ERR_ARG, "mi3_energies: null pointer");
    if (L < 2 || q < 1 || q > 255 || nseq > buflen)
        return fail(MI3_ERR_ARG, "mi3_energies: bad L/q/nseq");
    if (nseq == 0) return MI3_OK;
    if (ws_bytes < mi3_energies_workspace(nseq))
        return fail(MI3_ERR_WORKSPACE, "mi3_energies: workspace too small");
    if (!aligned(workspace, 8)) return fail(MI3_ERR_ALIGN, "mi3_energies: workspace alignment");
    cudaStream_t st = as_stream(stream);
    auto *acc = reinterpret_cast<unsigned long long *>(workspace);
    if (cudaMemsetAsync(acc, 0, (size_t)nseq * 8, st) != cudaSuccess)
        return check_launch("mi3_energies: memset");
    int rc = dispatch_energies<false>(J, seqmem, buflen, nseq, acc, L, q, nullptr, st);
    if (rc) return rc;
    k_energies_final<<<(nseq + 255) / 256, 256, 0, st>>>(acc, energies, nseq);
    return check_launch("mi3_energies: final");
}

// ---------------------------------------------------------------------------
// Allocation-free variant.  Some callers cannot allocate device memory at the
// point where they need energies: code running while a CUDA graph is being
// captured, hosts that hand the whole GPU to a pool they do not control, or
// foreign-language front ends that have no binding for a device allocator.
// For them the 64-bit accumulators live in a fixed array inside this library
// instead of a caller-provided workspace.  Capacity: MI3_ENERGIES_NOALLOC_MAX_SEQ
// sequences (8 bytes each, 8 MiB); every GPU on which the library's kernels are
// loaded holds the array until the process exits.
namespace mi3 {

static __device__ __align__(256) unsigned long long g_energies_noalloc_acc[MI3_ENERGIES_NOALLOC_MAX_SEQ];

// Device address of the array, per device.  The name of the array in host
// code is only a host-side handle, so it must not be passed to a kernel;
// cudaGetSymbolAddress gives the real device address for the device that is
// current when it runs.  The lookup is repeated on every call made outside
// stream capture (it is cheap), so a device reset or a new primary context
// never leaves a stale address behind; a call made during capture uses the
// address found by the last call made outside capture on that device.
static std::mutex g_noalloc_mutex;
static unsigned long long *g_noalloc_ptr[256] = {nullptr};

static int noalloc_scratch(cudaStream_t st, unsigned long long **out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 256)
        return fail(MI3_ERR_CUDA, std::string("mi3_energies_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(st, &cs);
    if (e != cudaSuccess)
        return fail(MI3_ERR_CUDA, std::string("mi3_energies_noalloc: cudaStreamIsCapturing: ") +
                                      cudaGetErrorString(e));
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (cs == cudaStreamCaptureStatusNone || !g_noalloc_ptr[dev]) {
        if (cs != cudaStreamCaptureStatusNone)
            return fail(MI3_ERR_ARG, "mi3_energies_noalloc: the first call on a device must not be made "
                                     "during stream capture");
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_energies_noalloc_acc);
        if (e != cudaSuccess || p == nullptr)
            return fail(MI3_ERR_CUDA,
                        std::string("mi3_energies_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_noalloc_ptr[dev] = static_cast<unsigned long long *>(p);
    }
    *out = g_noalloc_ptr[dev];
    return MI3_OK;
}

}  // namespace mi3

extern "C" int mi3_energies_noalloc(const float *J, const uint32_t *seqmem, uint32_t buflen, uint32_t nseq,
                                    float *energies, uint32_t L, uint32_t q, void *stream) {
    if (!J || !seqmem || !energies) return fail(MI3_ERR_ARG, "mi3_energies_noalloc: null pointer");
    if (L < 2 || q < 1 || q > 255 || nseq > buflen)
        return fail(MI3_ERR_ARG, "mi3_energies_noalloc: bad L/q/nseq");
    if (nseq > MI3_ENERGIES_NOALLOC_MAX_SEQ)
        return fail(MI3_ERR_ARG, "mi3_energies_noalloc: nseq " + std::to_string(nseq) +
                                     " exceeds the built-in scratch capacity of " +
                                     std::to_string((unsigned)MI3_ENERGIES_NOALLOC_MAX_SEQ) +
                                     " sequences; use mi3_energies with a workspace");
    // the address lookup comes first, so that any call -- a zero-size
    // warm-up included -- prepares the device for later calls under capture
    cudaStream_t st = as_stream(stream);
    unsigned long long *acc = nullptr;
    int rc = noalloc_scratch(st, &acc);
    if (rc) return rc;
    if (nseq == 0) return MI3_OK;
    // the accumulators keep the previous call's sums: clear the part used
    if (cudaMemsetAsync(acc, 0, (size_t)nseq * 8, st) != cudaSuccess)
        return check_launch("mi3_energies_noalloc: memset");
    rc = dispatch_energies<false>(J, seqmem, buflen, nseq, acc, L, q, nullptr, st);
    if (rc) return rc;
    k_energies_final<<<(nseq + 255) / 256, 256, 0, st>>>(acc, energies, nseq);
    return check_launch("mi3_energies_noalloc: final");
}

// ---------------------------------------------------------------------------
// Energies in the consensus gauge: the same values as mi3_energies (up to
// the rounding of the regauged couplings to float), with the pair work
// limited to the pairs where neither residue is its site's consensus.
extern "C" size_t mi3_energies_cons_workspace(uint32_t L, uint32_t q, uint32_t nseq) {
    const size_t acc = ((size_t)nseq * 8 + 255) & ~size_t(255);
    const size_t jc = ((size_t)npairs_of(L) * q * q * 4 + 255) & ~size_t(255);
    return acc + jc + (size_t)L * q * 8 + (size_t)L * 8;
}

extern "C" int mi3_energies_cons(const float *J, const uint32_t *seqmem, uint32_t buflen, uint32_t nseq,
                                 float *energies, uint32_t L, uint32_t q, const uint8_t *cons, void *workspace,
                                 size_t ws_bytes, void *stream) {
    if (!J || !seqmem || !energies || !cons || !workspace)
        return fail(MI3_ERR_ARG, "mi3_energies_cons: null pointer");
    if (L < 2 || q < 1 || q > 255 || nseq > buflen) return fail(MI3_ERR_ARG, "mi3_energies_cons: bad L/q/nseq");
    if ((size_t)(L * q + 1) * 8 > 200 * 1024) return fail(MI3_ERR_ARG, "mi3_energies_cons: L*q too large");
    if (nseq == 0) return MI3_OK;
    if (ws_bytes < mi3_energies_cons_workspace(L, q, nseq))
        return fail(MI3_ERR_WORKSPACE, "mi3_energies_cons: workspace too small");
    if (!aligned(workspace, 256)) return fail(MI3_ERR_ALIGN, "mi3_energies_cons: workspace must be 256B aligned");
    cudaStream_t st = as_stream(stream);
    unsigned char *ws = reinterpret_cast<unsigned char *>(workspace);
    auto *acc = reinterpret_cast<unsigned long long *>(ws);
    ws += ((size_t)nseq * 8 + 255) & ~size_t(255);
    float *Jc = reinterpret_cast<float *>(ws);
    ws += ((size_t)npairs_of(L) * q * q * 4 + 255) & ~size_t(255);
    double *h = reinterpret_cast<double *>(ws);
    double *cpart = h + (size_t)L * q;
    const uint64_t np = npairs_of(L);
    if (np > 0x7fffffffull) return fail(MI3_ERR_ARG, "mi3_energies_cons: L too large");
    k_cons_gauge<<<(uint32_t)np, 256, 0, st>>>(J, cons, Jc, L, q);
    int rc = check_launch("mi3_energies_cons: gauge");
    if (rc) return rc;
    k_cons_fields<<<L, 32, 0, st>>>(J, cons, h, cpart, L, q);
    rc = check_launch("mi3_energies_cons: fields");
    if (rc) return rc;
    if (cudaMemsetAsync(acc, 0, (size_t)nseq * 8, st) != cudaSuccess)
        return check_launch("mi3_energies_cons: memset");
    rc = dispatch_energies<true>(Jc, seqmem, buflen, nseq, acc, L, q, cons, st);
    if (rc) return rc;
    const size_t smem = (size_t)(L * q + 1) * 8;
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(k_energies_final_cons, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const uint32_t grid = std::min<uint32_t>((nseq + 255) / 256, 148 * 4);
    k_energies_final_cons<<<grid, 256, smem, st>>>(acc, seqmem, buflen, h, cpart, energies, nseq, L, q);
    return check_launch("mi3_energies_cons: final");
}
