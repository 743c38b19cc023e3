// equil.cu -- the round driver's equilibration test on the device.
//
// The reference decides that the walkers are equilibrated when the Spearman
// rank correlation between the energies at the latest checkpoint and those
// one and two checkpoints earlier is insignificant (scipy.stats.spearmanr,
// p > 0.02 for both; NewtonSteps.py:395-442).  spearmanr (scipy 1.18.1) is:
// average ranks of each vector (rankdata, ties get the mean of their
// positions), the Pearson correlation r of the two rank vectors, and the
// two-sided Student-t p-value of t = r sqrt((n-2) / ((1+r)(1-r))) with n-2
// degrees of freedom; a constant input gives r = NaN.  Since |t| grows with
// |r|, p > 0.02 is the same as |r| < r_crit with r_crit = t_c / sqrt(n - 2 +
// t_c^2), t_c the upper 1% point of that t distribution -- a number the host
// computes once per n.  Here:
//   mi3_rank_average   ranks of n floats (bitonic sort of (key, index)
//                      pairs, tie runs found by two prefix scans, average
//                      rank scattered back to the input order);
//   mi3_rank_corr      Pearson r of two rank vectors in FP64 (fixed-order
//                      reduction, so the result is deterministic);
//   mi3_equil_decide   the verdict |r1| < r_crit and |r2| < r_crit as an
//                      int32 flag in device memory (NaN fails).
#include <algorithm>
#include <cmath>

#include "common.cuh"

namespace mi3 {

constexpr uint32_t RK_THREADS = 1024;
constexpr uint32_t RK_TILE = 2 * RK_THREADS;  // elements sorted per block in shared memory
constexpr uint32_t RK_PAD_KEY = 0xffffffffu;   // sorts after every finite float

// Order-preserving map float -> uint32 (finite inputs); -0 and +0 are one
// value, as for a float comparison.
__device__ __forceinline__ uint32_t float_key(float x) {
    const uint32_t u = __float_as_uint(x == 0.0f ? 0.0f : x);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// (key, index) pairs compare by key, then index: a total order.
__device__ __forceinline__ bool pair_gt(uint32_t ka, uint32_t va, uint32_t kb, uint32_t vb) {
    return ka > kb || (ka == kb && va > vb);
}

__device__ __forceinline__ void cmp_swap(uint32_t &ka, uint32_t &va, uint32_t &kb, uint32_t &vb, bool asc) {
    if (pair_gt(ka, va, kb, vb) == asc) {
        uint32_t t = ka;
        ka = kb;
        kb = t;
        t = va;
        va = vb;
        vb = t;
    }
}

// The bitonic network's steps (k, j) with j < RK_TILE, for one tile in
// shared memory.  kmax = 0: every k from 2 to RK_TILE (the first pass over
// fresh input); otherwise only k = kmax (the tail of a global merge).
__device__ void tile_network(uint32_t *sk, uint32_t *sv, uint32_t base, uint32_t kmax) {
    const uint32_t k0 = kmax ? kmax : 2, k1 = kmax ? kmax : RK_TILE;
    for (uint32_t k = k0; k <= k1; k <<= 1) {
        for (uint32_t j = (k >> 1) < (RK_TILE >> 1) ? (k >> 1) : (RK_TILE >> 1); j > 0; j >>= 1) {
            const uint32_t t = threadIdx.x;
            const uint32_t i = 2 * j * (t / j) + (t % j), l = i + j;
            const bool asc = ((base + i) & k) == 0;
            cmp_swap(sk[i], sv[i], sk[l], sv[l], asc);
            __syncthreads();
        }
    }
}

__global__ void __launch_bounds__(RK_THREADS) k_rank_tiles(const float *__restrict__ x, uint32_t n,
                                                           uint32_t *keys, uint32_t *vals) {
    __shared__ uint32_t sk[RK_TILE], sv[RK_TILE];
    const uint32_t base = blockIdx.x * RK_TILE;
    for (uint32_t i = threadIdx.x; i < RK_TILE; i += RK_THREADS) {
        const uint32_t g = base + i;
        sk[i] = g < n ? float_key(x[g]) : RK_PAD_KEY;
        sv[i] = g;
    }
    __syncthreads();
    tile_network(sk, sv, base, 0);
    for (uint32_t i = threadIdx.x; i < RK_TILE; i += RK_THREADS) {
        keys[base + i] = sk[i];
        vals[base + i] = sv[i];
    }
}

// One global step (k, j >= RK_TILE): thread t compares pair (i, i + j).
__global__ void k_rank_global(uint32_t *keys, uint32_t *vals, uint32_t k, uint32_t j, uint32_t half) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= half) return;
    const uint32_t i = 2 * j * (t / j) + (t % j), l = i + j;
    uint32_t ka = keys[i], va = vals[i], kb = keys[l], vb = vals[l];
    cmp_swap(ka, va, kb, vb, (i & k) == 0);
    keys[i] = ka;
    vals[i] = va;
    keys[l] = kb;
    vals[l] = vb;
}

// Steps (k, j < RK_TILE) of a merge stage k > RK_TILE, one tile per block.
__global__ void __launch_bounds__(RK_THREADS) k_rank_merge(uint32_t *keys, uint32_t *vals, uint32_t k) {
    __shared__ uint32_t sk[RK_TILE], sv[RK_TILE];
    const uint32_t base = blockIdx.x * RK_TILE;
    for (uint32_t i = threadIdx.x; i < RK_TILE; i += RK_THREADS) {
        sk[i] = keys[base + i];
        sv[i] = vals[base + i];
    }
    __syncthreads();
    tile_network(sk, sv, base, k);
    for (uint32_t i = threadIdx.x; i < RK_TILE; i += RK_THREADS) {
        keys[base + i] = sk[i];
        vals[base + i] = sv[i];
    }
}

// Prefix maximum over positions (two levels: a block scan with its total,
// then the totals, then the carry) of: p where a run of equal sorted keys
// starts, else 0 (REV false: gives each position its run's first index);
// or, counting positions p' from the end, p' where a run ends (REV true:
// gives its run's last index as n - 1 - result).
constexpr uint32_t SC_THREADS = 1024, SC_PER = 4, SC_TILE = SC_THREADS * SC_PER;

template <bool REV>
__device__ __forceinline__ uint32_t run_mark(const uint32_t *keys, uint32_t n, uint32_t p) {
    // REV: p counts from the end; a run "starts" there when the next key
    // (towards the end) differs
    const uint32_t q = REV ? n - 1 - p : p;
    const bool edge = REV ? (q == n - 1 || keys[q] != keys[q + 1]) : (q == 0 || keys[q] != keys[q - 1]);
    return edge ? p : 0u;
}

template <bool REV>
__global__ void __launch_bounds__(SC_THREADS) k_scan_max_local(const uint32_t *__restrict__ keys, uint32_t n,
                                                               uint32_t *out, uint32_t *agg) {
    __shared__ uint32_t wtot[SC_THREADS / 32];
    const uint32_t base = blockIdx.x * SC_TILE + threadIdx.x * SC_PER;
    uint32_t v[SC_PER], run = 0;
#pragma unroll
    for (uint32_t e = 0; e < SC_PER; ++e) {
        const uint32_t p = base + e;
        v[e] = p < n ? run_mark<REV>(keys, n, p) : 0u;
        run = max(run, v[e]);
        v[e] = run;
    }
    // inclusive max-scan of the thread totals across the block
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = run;
#pragma unroll
    for (uint32_t o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x = max(x, y);
    }
    if (lane == 31) wtot[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < SC_THREADS / 32 ? wtot[lane] : 0u;
#pragma unroll
        for (uint32_t o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w = max(w, y);
        }
        if (lane < SC_THREADS / 32) wtot[lane] = w;
    }
    __syncthreads();
    uint32_t carry = __shfl_up_sync(0xffffffffu, x, 1);
    if (lane == 0) carry = 0;
    if (warp > 0) carry = max(carry, wtot[warp - 1]);
#pragma unroll
    for (uint32_t e = 0; e < SC_PER; ++e)
        if (base + e < n) out[base + e] = max(v[e], carry);
    if (threadIdx.x == 0) agg[blockIdx.x] = wtot[SC_THREADS / 32 - 1];  // the block's maximum
}

// Exclusive max-scan of the block totals (one block; nb <= SC_THREADS * SC_PER).
__global__ void __launch_bounds__(SC_THREADS) k_scan_max_aggs(uint32_t *agg, uint32_t nb) {
    if (threadIdx.x != 0) return;
    uint32_t run = 0;
    for (uint32_t b = 0; b < nb; ++b) {
        const uint32_t t = agg[b];
        agg[b] = run;
        run = max(run, t);
    }
}

__global__ void k_scan_max_apply(uint32_t *out, uint32_t n, const uint32_t *__restrict__ agg) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < n) out[p] = max(out[p], agg[p / SC_TILE]);
}

// rank (1-based, average over the tie run [lo, hi]) scattered to the input
// order
__global__ void k_rank_scatter(const uint32_t *__restrict__ vals, const uint32_t *__restrict__ lo,
                               const uint32_t *__restrict__ hirev, uint32_t n, float *ranks) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const uint32_t a = lo[p], b = n - 1 - hirev[n - 1 - p];
    ranks[vals[p]] = 0.5f * (float)(a + b) + 1.0f;  // exact: a + b < 2^24
}

// Pearson correlation of two rank vectors: per-block FP64 partial sums of
// (a-m)^2, (b-m)^2, (a-m)(b-m), m = (n+1)/2, then one thread in fixed order.
constexpr uint32_t PC_THREADS = 256, PC_BLOCKS = 296;

__global__ void __launch_bounds__(PC_THREADS) k_rank_corr_partial(const float *__restrict__ ra,
                                                                  const float *__restrict__ rb, uint32_t n,
                                                                  double *part) {
    __shared__ double s[3][PC_THREADS];
    const double m = 0.5 * ((double)n + 1.0);
    double aa = 0.0, bb = 0.0, ab = 0.0;
    for (uint32_t p = blockIdx.x * PC_THREADS + threadIdx.x; p < n; p += PC_BLOCKS * PC_THREADS) {
        const double a = (double)ra[p] - m, b = (double)rb[p] - m;
        aa += a * a;
        bb += b * b;
        ab += a * b;
    }
    s[0][threadIdx.x] = aa;
    s[1][threadIdx.x] = bb;
    s[2][threadIdx.x] = ab;
    __syncthreads();
    for (uint32_t o = PC_THREADS / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o)
            for (int c = 0; c < 3; ++c) s[c][threadIdx.x] += s[c][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int c = 0; c < 3; ++c) part[3 * blockIdx.x + c] = s[c][0];
}

__global__ void k_rank_corr_final(const double *__restrict__ part, double *r) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double aa = 0.0, bb = 0.0, ab = 0.0;
    for (uint32_t b = 0; b < PC_BLOCKS; ++b) {
        aa += part[3 * b];
        bb += part[3 * b + 1];
        ab += part[3 * b + 2];
    }
    // a constant input has no correlation (scipy: NaN)
    *r = (aa > 0.0 && bb > 0.0) ? ab / sqrt(aa * bb) : __longlong_as_double(0x7ff8000000000000ll);
}

__global__ void k_equil_decide(const double *r1, const double *r2, double rcrit, int32_t *flag) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double a = fabs(*r1), b = fabs(*r2);
    *flag = (a < rcrit && b < rcrit) ? 1 : 0;  // false for NaN
}

static uint32_t pow2_at_least(uint32_t n) {
    uint32_t p = RK_TILE;
    while (p < n) p <<= 1;
    return p;
}

}  // namespace mi3

using namespace mi3;

extern "C" size_t mi3_rank_workspace(uint32_t n) {
    if (n == 0 || n >= (1u << 23)) return 0;
    const size_t P = pow2_at_least(n);
    const size_t nb = (n + SC_TILE - 1) / SC_TILE;
    return 2 * P * 4 + 2 * (size_t)n * 4 + 256 + nb * 4;
}

extern "C" int mi3_rank_average(const float *x, uint32_t n, float *ranks, void *workspace, size_t ws_bytes,
                                void *stream) {
    if (!x || !ranks || !workspace) return fail(MI3_ERR_ARG, "mi3_rank_average: null pointer");
    if (n == 0 || n >= (1u << 23)) return fail(MI3_ERR_ARG, "mi3_rank_average: need 0 < n < 2^23");
    if (ws_bytes < mi3_rank_workspace(n)) return fail(MI3_ERR_WORKSPACE, "mi3_rank_average: workspace too small");
    if (!aligned(workspace, 16)) return fail(MI3_ERR_ALIGN, "mi3_rank_average: workspace must be 16B aligned");
    cudaStream_t st = as_stream(stream);
    const uint32_t P = pow2_at_least(n);
    uint32_t *keys = reinterpret_cast<uint32_t *>(workspace);
    uint32_t *vals = keys + P;
    uint32_t *lo = vals + P;
    uint32_t *hirev = lo + n;
    uint32_t *agg = reinterpret_cast<uint32_t *>(reinterpret_cast<unsigned char *>(hirev + n) + 256);
    k_rank_tiles<<<P / RK_TILE, RK_THREADS, 0, st>>>(x, n, keys, vals);
    const uint32_t half = P / 2;
    for (uint32_t k = 2 * RK_TILE; k <= P; k <<= 1) {
        for (uint32_t j = k >> 1; j >= RK_TILE; j >>= 1)
            k_rank_global<<<(half + 255) / 256, 256, 0, st>>>(keys, vals, k, j, half);
        k_rank_merge<<<P / RK_TILE, RK_THREADS, 0, st>>>(keys, vals, k);
    }
    const uint32_t nb = (n + SC_TILE - 1) / SC_TILE;
    k_scan_max_local<false><<<nb, SC_THREADS, 0, st>>>(keys, n, lo, agg);
    k_scan_max_aggs<<<1, 32, 0, st>>>(agg, nb);
    k_scan_max_apply<<<(n + 255) / 256, 256, 0, st>>>(lo, n, agg);
    k_scan_max_local<true><<<nb, SC_THREADS, 0, st>>>(keys, n, hirev, agg);
    k_scan_max_aggs<<<1, 32, 0, st>>>(agg, nb);
    k_scan_max_apply<<<(n + 255) / 256, 256, 0, st>>>(hirev, n, agg);
    k_rank_scatter<<<(n + 255) / 256, 256, 0, st>>>(vals, lo, hirev, n, ranks);
    return check_launch("mi3_rank_average");
}

extern "C" size_t mi3_rank_corr_workspace(void) { return (size_t)PC_BLOCKS * 3 * 8; }

extern "C" int mi3_rank_corr(const float *ranks_a, const float *ranks_b, uint32_t n, double *r, void *workspace,
                             size_t ws_bytes, void *stream) {
    if (!ranks_a || !ranks_b || !r || !workspace) return fail(MI3_ERR_ARG, "mi3_rank_corr: null pointer");
    if (n < 2) return fail(MI3_ERR_ARG, "mi3_rank_corr: need n >= 2");
    if (ws_bytes < mi3_rank_corr_workspace()) return fail(MI3_ERR_WORKSPACE, "mi3_rank_corr: workspace too small");
    if (!aligned(workspace, 8)) return fail(MI3_ERR_ALIGN, "mi3_rank_corr: workspace must be 8B aligned");
    cudaStream_t st = as_stream(stream);
    double *part = reinterpret_cast<double *>(workspace);
    k_rank_corr_partial<<<PC_BLOCKS, PC_THREADS, 0, st>>>(ranks_a, ranks_b, n, part);
    k_rank_corr_final<<<1, 32, 0, st>>>(part, r);
    return check_launch("mi3_rank_corr");
}

extern "C" int mi3_equil_decide(const double *r1, const double *r2, double rcrit, int32_t *flag, void *stream) {
    if (!r1 || !r2 || !flag) return fail(MI3_ERR_ARG, "mi3_equil_decide: null pointer");
    k_equil_decide<<<1, 32, 0, as_stream(stream)>>>(r1, r2, rcrit, flag);
    return check_launch("mi3_equil_decide");
}
