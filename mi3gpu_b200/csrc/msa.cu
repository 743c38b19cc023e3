// msa.cu -- walkers as the text lines of an MSA file, in the format the
// reference writes and reads (mi3gpu/utils/seqload.py: writeSeqs
// seqload.py:378-411, loadSeqs seqload.py:91-133 and 196-352), formatted and
// parsed on the device so walkers go to and from files without a host
// transpose or table lookup.
//
// Both kernels are HBM streams (4 bytes per packed word one way, one byte
// per text character the other).  A CTA works on tiles of T walkers: the
// packed words of a tile are (SWORDS, T) columns of the walker-minor
// buffer, read or written coalesced along the walker axis; the tile's text
// is T consecutive lines, a contiguous run of bytes that starts on a
// 16-byte boundary (T is a multiple of 16), moved as 16-byte vectors.  The
// transpose between the two sits in shared memory (words and lines back to
// back); global loads are unrolled so each thread has several in flight.
#include <cstring>

#include "common.cuh"

namespace mi3 {

struct Alphabet {
    uint8_t c[256];
};

constexpr uint32_t MSA_THREADS = 256;
constexpr uint32_t MSA_SMEM_TARGET = 48 * 1024;   // preferred tile footprint
constexpr uint32_t MSA_SMEM_MAX = 200 * 1024;     // largest tile footprint

__host__ __device__ inline uint32_t msa_words_bytes(uint32_t SW, uint32_t T) { return SW * T * 4; }
__host__ __device__ inline uint32_t msa_lines_bytes(uint32_t line_len, uint32_t T) {
    return (T * line_len + 15) & ~15u;
}

// Largest power-of-two tile (16..128 walkers) whose staging fits the target
// footprint, else the largest that fits at all; 0 if none does.
static uint32_t msa_tile(uint32_t SW, uint32_t line_len) {
    for (uint32_t lim : {MSA_SMEM_TARGET, MSA_SMEM_MAX})
        for (uint32_t T = 128; T >= 16; T >>= 1)
            if ((uint64_t)msa_words_bytes(SW, T) + msa_lines_bytes(line_len, T) <= lim) return T;
    return 0;
}

// Copy nbytes from src to dst, both 16-byte aligned, with the CTA's
// threads; each thread has U 16-byte loads in flight before it stores.
__device__ __forceinline__ void copy_bytes_v16(uint8_t *__restrict__ dst, const uint8_t *__restrict__ src,
                                               uint32_t nbytes) {
    constexpr uint32_t U = 4;
    const uint32_t nvec = nbytes >> 4;
    const uint4 *s4 = reinterpret_cast<const uint4 *>(src);
    uint4 *d4 = reinterpret_cast<uint4 *>(dst);
    for (uint32_t base = 0; base < nvec; base += U * blockDim.x) {
        uint4 v[U];
#pragma unroll
        for (uint32_t k = 0; k < U; ++k) {
            const uint32_t i = base + k * blockDim.x + threadIdx.x;
            if (i < nvec) v[k] = s4[i];
        }
#pragma unroll
        for (uint32_t k = 0; k < U; ++k) {
            const uint32_t i = base + k * blockDim.x + threadIdx.x;
            if (i < nvec) d4[i] = v[k];
        }
    }
    for (uint32_t p = (nvec << 4) + threadIdx.x; p < nbytes; p += blockDim.x) dst[p] = src[p];
}

// The (SWORDS, nt) packed words of walkers [j0, j0+nt) into words[w*T+t];
// each thread has U loads in flight before it stores.
template <uint32_t T>
__device__ __forceinline__ void load_words(uint32_t *__restrict__ words, const uint32_t *__restrict__ seqmem,
                                           uint32_t buflen, uint32_t j0, uint32_t nt, uint32_t SW) {
    constexpr uint32_t LOG_T = __builtin_ctz(T), U = 8;
    const uint32_t n = SW * T;
    for (uint32_t base = 0; base < n; base += U * blockDim.x) {
        uint32_t v[U];
#pragma unroll
        for (uint32_t k = 0; k < U; ++k) {
            const uint32_t i = base + k * blockDim.x + threadIdx.x;
            const uint32_t w = i >> LOG_T, t = i & (T - 1);
            v[k] = (i < n && t < nt) ? __ldg(seqmem + (size_t)w * buflen + j0 + t) : 0u;
        }
#pragma unroll
        for (uint32_t k = 0; k < U; ++k) {
            const uint32_t i = base + k * blockDim.x + threadIdx.x;
            if (i < n) words[i] = v[k];
        }
    }
}

// Index mapping shared by every phase: element i of a tile is (word w =
// i / T, walker t = i % T), with T a power of two, so consecutive threads
// take consecutive walkers: global words are read or written coalesced,
// shared words words[w*T+t] are conflict free, and the text bytes of
// consecutive threads sit one line apart (a stride that spreads over the
// banks unless the line length is a multiple of 128).
template <uint32_t T>
__global__ void __launch_bounds__(MSA_THREADS) k_seqs_to_text(const uint32_t *__restrict__ seqmem, uint32_t buflen,
                                                              uint32_t nseq, uint32_t L, Alphabet alpha,
                                                              uint32_t nalpha, uint8_t *__restrict__ text,
                                                              int32_t *status) {
    constexpr uint32_t LOG_T = __builtin_ctz(T);
    extern __shared__ __align__(16) uint8_t smem[];
    const uint32_t SW = (L - 1) / 4 + 1, LL = L + 1;
    uint8_t *lines = smem;                                                         // [T][L+1]
    uint32_t *words = reinterpret_cast<uint32_t *>(smem + msa_lines_bytes(LL, T));  // [SW][T]
    __shared__ uint8_t table[256];
    for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x) table[i] = alpha.c[i];
    bool bad = false;
    const uint32_t ntiles = (nseq + T - 1) / T;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint32_t j0 = tile * T, nt = min(T, nseq - j0);
        __syncthreads();  // the previous tile's lines are written out
        load_words<T>(words, seqmem, buflen, j0, nt, SW);
        __syncthreads();
        // one packed word -> four characters of one line; the thread that
        // holds a line's last word also ends the line
        for (uint32_t i = threadIdx.x; i < SW * T; i += blockDim.x) {
            const uint32_t w = i >> LOG_T, t = i & (T - 1);
            if (t >= nt) continue;
            const uint32_t x = words[i];
            uint8_t *ln = lines + t * LL;
#pragma unroll
            for (uint32_t b = 0; b < 4; ++b) {
                const uint32_t c = 4 * w + b;
                if (c < L) {
                    const uint32_t r = (x >> (8 * b)) & 0xffu;
                    bad |= r >= nalpha;
                    ln[c] = r < nalpha ? table[r] : (uint8_t)'?';
                }
            }
            if (w == SW - 1) ln[L] = '\n';
        }
        __syncthreads();
        copy_bytes_v16(text + (size_t)j0 * LL, lines, nt * LL);
    }
    if (bad) report(status, ST_BAD_INPUT);
}

template <uint32_t T>
__global__ void __launch_bounds__(MSA_THREADS) k_text_to_seqs(const uint8_t *__restrict__ text, uint32_t nseq,
                                                              uint32_t line_len, uint32_t id_len, uint32_t L,
                                                              Alphabet lookup, uint32_t *__restrict__ seqmem,
                                                              uint32_t buflen, uint32_t n0,
                                                              unsigned long long *first_bad) {
    constexpr uint32_t LOG_T = __builtin_ctz(T);
    extern __shared__ __align__(16) uint8_t smem[];
    const uint32_t SW = (L - 1) / 4 + 1;
    uint8_t *lines = smem;                                                               // [T][line_len]
    uint32_t *words = reinterpret_cast<uint32_t *>(smem + msa_lines_bytes(line_len, T));  // [SW][T]
    __shared__ uint8_t table[256];
    for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x) table[i] = lookup.c[i];
    const uint32_t ntiles = (nseq + T - 1) / T;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint32_t j0 = tile * T, nt = min(T, nseq - j0);
        __syncthreads();  // the previous tile's words are stored
        copy_bytes_v16(lines, text + (size_t)j0 * line_len, nt * line_len);
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < SW * T; i += blockDim.x) {
            const uint32_t w = i >> LOG_T, t = i & (T - 1);
            if (t >= nt) continue;
            const uint8_t *ln = lines + t * line_len;
            bool ok = true;
            if (w == 0) ok = ln[line_len - 1] == '\n' && (id_len == 0 || ln[id_len - 1] == ' ');
            uint32_t x = 0;
#pragma unroll
            for (uint32_t b = 0; b < 4; ++b) {
                const uint32_t c = 4 * w + b;
                if (c < L) {
                    const uint32_t r = table[ln[id_len + c]];
                    ok &= r != 0xffu;
                    x |= (r & 0xffu) << (8 * b);
                }
            }
            if (!ok) atomicMin(first_bad, (unsigned long long)(j0 + t));
            words[i] = x;
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < SW * T; i += blockDim.x) {
            const uint32_t w = i >> LOG_T, t = i & (T - 1);
            if (t < nt) seqmem[(size_t)w * buflen + n0 + j0 + t] = words[i];
        }
    }
}

static int msa_launch_setup(const void *kernel, uint32_t smem) {
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return fail(MI3_ERR_CUDA, std::string("msa smem attribute: ") + cudaGetErrorString(e));
    }
    return MI3_OK;
}

static uint32_t msa_grid(uint32_t ntiles, uint32_t smem) {
    const uint32_t per_sm = std::max<uint32_t>(1, std::min<uint32_t>(8, (227 * 1024) / (smem + 1024)));
    return std::max<uint32_t>(1, std::min<uint32_t>(ntiles, 148 * per_sm));
}

}  // namespace mi3

extern "C" int mi3_seqs_to_text(const uint32_t *seqmem, uint32_t buflen, uint32_t nseq, uint32_t L,
                                const char *alpha, uint32_t nalpha, uint8_t *text, int32_t *status, void *stream) {
    using namespace mi3;
    if (!seqmem || !text || !alpha || !status) return fail(MI3_ERR_ARG, "mi3_seqs_to_text: null pointer");
    if (L == 0 || nseq > buflen || nalpha == 0 || nalpha > 256)
        return fail(MI3_ERR_ARG, "mi3_seqs_to_text: need L > 0, nseq <= buflen, 1 <= nalpha <= 256");
    if (!aligned(text, 16)) return fail(MI3_ERR_ALIGN, "mi3_seqs_to_text: text must be 16-byte aligned");
    if (nseq == 0) return MI3_OK;
    const uint32_t SW = swords_of(L), T = msa_tile(SW, L + 1);
    if (T == 0) return fail(MI3_ERR_ARG, "mi3_seqs_to_text: L too large");
    Alphabet a{};
    for (uint32_t i = 0; i < nalpha; ++i) a.c[i] = (uint8_t)alpha[i];
    const uint32_t smem = msa_lines_bytes(L + 1, T) + msa_words_bytes(SW, T);
    auto launch = [&](auto kernel) -> int {
        if (int rc = msa_launch_setup((const void *)kernel, smem)) return rc;
        kernel<<<msa_grid((nseq + T - 1) / T, smem), MSA_THREADS, smem, as_stream(stream)>>>(
            seqmem, buflen, nseq, L, a, nalpha, text, status);
        return check_launch("mi3_seqs_to_text");
    };
    switch (T) {
        case 128: return launch(k_seqs_to_text<128>);
        case 64: return launch(k_seqs_to_text<64>);
        case 32: return launch(k_seqs_to_text<32>);
        default: return launch(k_seqs_to_text<16>);
    }
}

extern "C" int mi3_text_to_seqs(const uint8_t *text, uint32_t nseq, uint32_t line_len, uint32_t id_len, uint32_t L,
                                const char *alpha, uint32_t nalpha, uint32_t *seqmem, uint32_t buflen, uint32_t n0,
                                uint64_t *first_bad, void *stream) {
    using namespace mi3;
    if (!text || !seqmem || !alpha || !first_bad) return fail(MI3_ERR_ARG, "mi3_text_to_seqs: null pointer");
    if (L == 0 || nalpha == 0 || nalpha > 255 || line_len != id_len + L + 1 || (uint64_t)n0 + nseq > buflen)
        return fail(MI3_ERR_ARG,
                    "mi3_text_to_seqs: need L > 0, 1 <= nalpha <= 255, line_len = id_len + L + 1, "
                    "n0 + nseq <= buflen");
    if (!aligned(text, 16)) return fail(MI3_ERR_ALIGN, "mi3_text_to_seqs: text must be 16-byte aligned");
    cudaError_t e = cudaMemsetAsync(first_bad, 0xff, sizeof(uint64_t), as_stream(stream));
    if (e != cudaSuccess) return fail(MI3_ERR_CUDA, std::string("mi3_text_to_seqs: ") + cudaGetErrorString(e));
    if (nseq == 0) return MI3_OK;
    const uint32_t SW = swords_of(L), T = msa_tile(SW, line_len);
    if (T == 0) return fail(MI3_ERR_ARG, "mi3_text_to_seqs: lines too long");
    // ASCII -> residue index; later alphabet letters win, as numpy's
    // fancy assignment does in the reference's table (seqload.py:205-206)
    Alphabet lut;
    memset(lut.c, 0xff, sizeof(lut.c));
    for (uint32_t i = 0; i < nalpha; ++i) lut.c[(uint8_t)alpha[i]] = (uint8_t)i;
    const uint32_t smem = msa_lines_bytes(line_len, T) + msa_words_bytes(SW, T);
    auto launch = [&](auto kernel) -> int {
        if (int rc = msa_launch_setup((const void *)kernel, smem)) return rc;
        kernel<<<msa_grid((nseq + T - 1) / T, smem), MSA_THREADS, smem, as_stream(stream)>>>(
            text, nseq, line_len, id_len, L, lut, seqmem, buflen, n0,
            reinterpret_cast<unsigned long long *>(first_bad));
        return check_launch("mi3_text_to_seqs");
    };
    switch (T) {
        case 128: return launch(k_text_to_seqs<128>);
        case 64: return launch(k_text_to_seqs<64>);
        case 32: return launch(k_text_to_seqs<32>);
        default: return launch(k_text_to_seqs<16>);
    }
}
