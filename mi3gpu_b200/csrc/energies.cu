// energies.cu -- Potts energies E(s) = sum_{i<j} J_ij(s_i, s_j).
//
// Slice-tiled (tiling.cuh): a CTA holds the couplings of one block pair in
// shared memory and streams a chunk of sequences through it; each thread
// sums its sequence's B*B gathered couplings in double and adds the slice
// total to a per-sequence 64-bit fixed-point accumulator (scale 2^40) with an
// integer atomic.  Integer addition is associative, so the result does not
// depend on CTA order: energies are deterministic, and accurate to ~1e-12
// absolute before the final rounding to float.  The reference sums each
// sequence serially with Kahan compensation in float (getEnergiesf,
// mcmc.cl:249-336); this result is at least as accurate.
#include <mutex>

#include "tiling.cuh"

namespace mi3 {

constexpr double FIX_SCALE = 1099511627776.0;  // 2^40
constexpr double FIX_INV = 1.0 / 1099511627776.0;

template <int B>
__global__ void __launch_bounds__(512) k_energies(const float *__restrict__ J,
                                                  const uint32_t *__restrict__ seq, uint32_t buflen,
                                                  uint32_t nseq, unsigned long long *acc, uint32_t L,
                                                  uint32_t q, SliceGeom g) {
    extern __shared__ __align__(16) float js[];  // [B*B][q*q]
    const uint32_t qq = q * q;
    const uint32_t s = blockIdx.x % g.nslices;
    const uint32_t chunk = blockIdx.x / g.nslices;
    uint32_t bi, bj;
    slice_coords(s, g.nb, bi, bj);
    const uint32_t i0 = bi * B, j0 = bj * B;

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
    __syncthreads();

    const uint32_t swords = (L - 1) / 4 + 1;
    const uint32_t nbeg = chunk * g.chunk;
    const uint32_t nend = min(nseq, nbeg + g.chunk);
    // two sequences per thread: two independent gather/add chains in flight
    for (uint32_t n = nbeg + threadIdx.x; n < nend; n += 2 * blockDim.x) {
        const uint32_t n2 = n + blockDim.x;
        const bool two = n2 < nend;
        uint32_t wI[B / 4], wJ[B / 4], vI[B / 4], vJ[B / 4];
        load_block_words<B>(seq, buflen, n, bi, swords, wI);
        load_block_words<B>(seq, buflen, n, bj, swords, wJ);
        load_block_words<B>(seq, buflen, two ? n2 : n, bi, swords, vI);
        load_block_words<B>(seq, buflen, two ? n2 : n, bj, swords, vJ);
        double e1 = 0.0, e2 = 0.0;
#pragma unroll
        for (int ii = 0; ii < B; ++ii) {
            uint32_t i = i0 + ii;
            if (i >= L) break;
            const float *row1 = js + (size_t)ii * B * qq + block_byte<B>(wI, ii, q - 1) * q;
            const float *row2 = js + (size_t)ii * B * qq + block_byte<B>(vI, ii, q - 1) * q;
#pragma unroll
            for (int jj = 0; jj < B; ++jj) {
                uint32_t j = j0 + jj;
                if (j < L && j > i) {
                    e1 += (double)row1[(size_t)jj * qq + block_byte<B>(wJ, jj, q - 1)];
                    e2 += (double)row2[(size_t)jj * qq + block_byte<B>(vJ, jj, q - 1)];
                }
            }
        }
        atomicAdd(&acc[n], (unsigned long long)__double2ll_rn(e1 * FIX_SCALE));
        if (two) atomicAdd(&acc[n2], (unsigned long long)__double2ll_rn(e2 * FIX_SCALE));
    }
}

__global__ void k_energies_final(const unsigned long long *__restrict__ acc, float *E, uint32_t n) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) E[k] = (float)((double)(long long)acc[k] * FIX_INV);
}

template <int B>
static int launch_energies(const float *J, const uint32_t *seq, uint32_t buflen, uint32_t nseq,
                           unsigned long long *acc, uint32_t L, uint32_t q, cudaStream_t st) {
    SliceGeom g = make_geom(L, B, nseq, 148 * 8, 2048);
    size_t smem = (size_t)B * B * q * q * 4;
    cudaFuncSetAttribute(k_energies<B>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    uint64_t nblk = (uint64_t)g.nslices * g.nchunks;
    if (nblk > 0x7fffffffull) return fail(MI3_ERR_ARG, "mi3_energies: grid too large");
    k_energies<B><<<(uint32_t)nblk, 512, smem, st>>>(J, seq, buflen, nseq, acc, L, q, g);
    return check_launch("mi3_energies");
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
    uint32_t B = pick_block(q, 116 * 1024);
    int rc;
    switch (B) {
        case 32: rc = launch_energies<32>(J, seqmem, buflen, nseq, acc, L, q, st); break;
        case 16: rc = launch_energies<16>(J, seqmem, buflen, nseq, acc, L, q, st); break;
        case 8: rc = launch_energies<8>(J, seqmem, buflen, nseq, acc, L, q, st); break;
        case 4: rc = launch_energies<4>(J, seqmem, buflen, nseq, acc, L, q, st); break;
        default: return fail(MI3_ERR_ARG, "mi3_energies: q too large");
    }
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

// Device address of the array, looked up once per device.  The name of the
// array in host code is only a host-side handle, so it must not be passed to
// a kernel; cudaGetSymbolAddress gives the real device address for the device
// that is current when it runs.
static std::mutex g_noalloc_mutex;
static unsigned long long *g_noalloc_ptr[256] = {nullptr};

static int noalloc_scratch(unsigned long long **out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 256)
        return fail(MI3_ERR_CUDA, std::string("mi3_energies_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
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
    if (nseq == 0) return MI3_OK;
    unsigned long long *acc = nullptr;
    int rc = noalloc_scratch(&acc);
    if (rc) return rc;
    cudaStream_t st = as_stream(stream);
    // the accumulators keep the previous call's sums: clear the part used
    if (cudaMemsetAsync(acc, 0, (size_t)nseq * 8, st) != cudaSuccess)
        return check_launch("mi3_energies_noalloc: memset");
    switch (pick_block(q, 116 * 1024)) {
        case 32: rc = launch_energies<32>(J, seqmem, buflen, nseq, acc, L, q, st); break;
        case 16: rc = launch_energies<16>(J, seqmem, buflen, nseq, acc, L, q, st); break;
        case 8: rc = launch_energies<8>(J, seqmem, buflen, nseq, acc, L, q, st); break;
        case 4: rc = launch_energies<4>(J, seqmem, buflen, nseq, acc, L, q, st); break;
        default: return fail(MI3_ERR_ARG, "mi3_energies_noalloc: q too large");
    }
    if (rc) return rc;
    k_energies_final<<<(nseq + 255) / 256, 256, 0, st>>>(acc, energies, nseq);
    return check_launch("mi3_energies_noalloc: final");
}
