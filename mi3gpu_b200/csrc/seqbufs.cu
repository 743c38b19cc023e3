// seqbufs.cu -- operations between sequence buffers: the subsequence splice
// of the reference's subsequence-frequency mode (copySubseq,
// mcmc.cl:99-122; markPos, mcmcGPU.py:919-925).
#include "common.cuh"

namespace mi3 {

// Every sequence n of the large buffer takes, at the marked sites, the
// residues of sequence `seqind` of the small buffer: per packed word a
// byte-masked merge, (large & ~m) | (sub & m).  One thread per (word,
// sequence), consecutive threads on consecutive sequences (coalesced);
// words without a marked site are not touched.
__global__ void k_copy_subseq(const uint32_t *__restrict__ small, uint32_t nsmall, uint32_t seqind,
                              const uint8_t *__restrict__ marks, uint32_t *__restrict__ large, uint32_t nlarge,
                              uint32_t L) {
    const uint32_t w = blockIdx.y;
    const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t m = 0;
#pragma unroll
    for (uint32_t b = 0; b < 4; ++b)
        if (4 * w + b < L && marks[4 * w + b]) m |= 0xffu << (8 * b);
    if (m == 0 || n >= nlarge) return;
    const uint32_t sub = __ldg(small + (size_t)w * nsmall + seqind);
    uint32_t *p = large + (size_t)w * nlarge + n;
    *p = (*p & ~m) | (sub & m);
}

}  // namespace mi3

extern "C" int mi3_copy_subseq(const uint32_t *small, uint32_t nsmall, uint32_t seqind, const uint8_t *marks,
                               uint32_t *large, uint32_t nlarge, uint32_t L, void *stream) {
    using namespace mi3;
    if (!small || !marks || !large) return fail(MI3_ERR_ARG, "mi3_copy_subseq: null pointer");
    if (L == 0 || seqind >= nsmall) return fail(MI3_ERR_ARG, "mi3_copy_subseq: need L > 0 and seqind < nsmall");
    if (nlarge == 0) return MI3_OK;
    dim3 grid((nlarge + 255) / 256, swords_of(L));
    k_copy_subseq<<<grid, 256, 0, as_stream(stream)>>>(small, nsmall, seqind, marks, large, nlarge, L);
    return check_launch("mi3_copy_subseq");
}
