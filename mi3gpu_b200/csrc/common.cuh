// common.cuh -- shared device helpers for libmi3b200 (sm_100a).
//
// MWC64X generator steps, the Metropolis acceptance test, mbarrier / bulk-copy
// wrappers with bounded waits, and host-side error plumbing for the C ABI.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <algorithm>
#include <string>

#include "../../include/mi3b200.h"

namespace mi3 {

// ---------------------------------------------------------------- host errors
void set_error(const std::string &msg);
int fail(int code, const std::string &msg);
int check_launch(const char *what);

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }
inline bool aligned(const void *p, size_t a) { return (reinterpret_cast<uintptr_t>(p) % a) == 0; }
inline uint64_t npairs_of(uint32_t L) { return (uint64_t)L * (L - 1) / 2; }
inline uint32_t swords_of(uint32_t L) { return (L - 1) / 4 + 1; }

// Floats per row of the unpacked coupling layout: L blocks of q*q, padded to a
// multiple of 4 floats so that every row and every 4-site chunk of a row
// starts on a 16-byte boundary (bulk-copy alignment).
inline uint64_t jrow_stride(uint32_t L, uint32_t q) {
    uint64_t n = (uint64_t)L * q * q;
    return (n + 3) & ~uint64_t(3);
}

// -------------------------------------------------------------- MWC64X (RNG)
// Multiply-with-carry generator, multiplier A, modulus A*2^32-1 (the MWC64X
// generator of the reference, mwc64x_rng.cl:17-27).  One walker holds two
// independent lanes: state image {x0, x1, c0, c1}.
constexpr uint32_t MWC_A = 4294883355u;

__device__ __forceinline__ void mwc_step(uint32_t &x, uint32_t &c) {
    uint32_t xn = MWC_A * x + c;
    uint32_t carry = (xn < c) ? 1u : 0u;
    uint32_t cn = __umulhi(MWC_A, x) + carry;
    x = xn;
    c = cn;
}

struct Rng2 {
    uint32_t x0, x1, c0, c1;
};

__device__ __forceinline__ void rng_next2(Rng2 &s, uint32_t &r0, uint32_t &r1) {
    r0 = s.x0 ^ s.c0;
    r1 = s.x1 ^ s.c1;
    mwc_step(s.x0, s.c0);
    mwc_step(s.x1, s.c1);
}

__device__ __forceinline__ float uniform_map(uint32_t i) {
    return (float)(i >> 8) * 0x1.0p-24f;
}

// Metropolis test exp(x) > u with exp rounded correctly to float.  expf has a
// documented maximum error of 2 ulp, so when it lands further than 2^-19
// relative from u its verdict equals the correctly rounded one; otherwise the
// double exp, rounded to float, decides.  The CPU oracle takes the double
// route every time, so both make the same decision.
__device__ __forceinline__ bool accept_exp(float x, float u) {
    if (x >= 0.0f) return true;
    float e = expf(x);
    if (u > 0.0f && e >= 0x1p-100f) {
        float tol = u * 0x1p-19f;
        if (e > u + tol) return true;
        if (e < u - tol) return false;
    }
    return (float)exp((double)x) > u;
}

// ---------------------------------------------------------- sequence bytes
__device__ __forceinline__ uint32_t getbyte(uint32_t w, uint32_t k) {
    return (w >> (8u * k)) & 0xffu;
}
__device__ __forceinline__ uint32_t setbyte(uint32_t w, uint32_t k, uint32_t v) {
    uint32_t sh = 8u * k;
    return (w & ~(0xffu << sh)) | ((v & 0xffu) << sh);
}

// ------------------------------------------------------- mbarrier / bulk copy
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count));
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Wait for the phase with parity `parity` of `bar` to complete, giving up
// after `limit_ns` nanoseconds or as soon as *abort is set.  Returns false on
// give-up.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity,
                                                  const volatile int *abort, uint64_t limit_ns) {
#pragma unroll 1
    for (int i = 0; i < 32; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    uint64_t t0 = globaltimer_ns();
#pragma unroll 1
    while (true) {
        if (mbar_try_wait(bar, parity)) return true;
        if (abort && *abort) return false;
        if (globaltimer_ns() - t0 > limit_ns) return false;
    }
}

// 1-D bulk copy global -> shared, completion counted on `bar` in bytes.
// dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// Status word codes written by kernels (first error wins).
constexpr int ST_TIMEOUT_FULL = 1;
constexpr int ST_TIMEOUT_EMPTY = 2;
constexpr int ST_BAD_INPUT = 3;

__device__ __forceinline__ void report(int32_t *status, int code) {
    if (status) atomicCAS(reinterpret_cast<int *>(status), 0, code);
}

constexpr uint64_t WAIT_LIMIT_NS = 4000000000ull;  // 4 s per wait

}  // namespace mi3
