// newton.cu -- the quasi-Newton coupling update and the Zwanzig reweighting
// statistics (NewtonSteps.iterNewton, NewtonSteps.py:159-268).
//
//   mi3_update_j         updatedJ           (mcmc.cl:829-843)
//   mi3_reg_l1z / l2z    reg_l1z / reg_l2z  (mcmc.cl:845-902, zeroGauge :764-822)
//   mi3_min_floats       minFloats          (mcmc.cl:558-584)
//   mi3_dE_to_weights    dE_to_weights      (mcmc.cl:624-633)
//   mi3_fixed_beta_weights                  (mcmc.cl:635-644)
//   mi3_weight_stats     weight_stats       (mcmc.cl:586-622), in double
//   mi3_weights_fused    dE -> (weights, min dE, sums) in one pass
//   mi3_add_float_bufs   addFloatBufs       (mcmc.cl:720-727)
//
// Reductions over walkers run as a fixed grid of CTAs that write partials to
// a workspace; the last CTA to finish (ticket counter) combines them in a
// fixed order, so sums are deterministic.
#include "common.cuh"

namespace mi3 {

__global__ void k_update_j(const float *__restrict__ bt, const float *__restrict__ bi, float gamma,
                           float pc, const float *Ji, float *Jo, uint64_t n) {
    uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) Jo[k] = Ji[k] - gamma * (bt[k] - bi[k]) / (bi[k] + pc);
}

__device__ __forceinline__ float ocl_sign(float x) {
    if (x > 0.0f) return 1.0f;
    if (x < 0.0f) return -1.0f;
    if (x != x) return 0.0f;
    return x;
}

// Odd-aware tree over the q columns of each row of the q*q scratch block
// (the row loops of zeroGauge, mcmc.cl:772-781).  One warp.
__device__ __forceinline__ void rows_tree(float *sc, uint32_t q, uint32_t lane) {
    const uint32_t qq = q * q;
    uint32_t m = q;
    while (m > 1) {
        uint32_t odd = m & 1;
        m = (m + 1) >> 1;
        for (uint32_t li = lane; li < qq; li += 32)
            if (li % q < m - odd) sc[li] = sc[li] + sc[li + m];
        __syncwarp();
    }
}

// reg_l1z (L2=false) / reg_l2z (L2=true): one warp per pair block.
template <bool L2>
__global__ void k_reg_lz(const float *__restrict__ bi, float gamma, float pc, float lJ,
                         const float *__restrict__ J, float *dJ, uint64_t npairs, uint32_t q) {
    extern __shared__ float sm[];
    const uint32_t qq = q * q;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t wpb = blockDim.x >> 5;
    float *sc = sm + warp * (qq + 2 * q + 2);  // [q*q scratch][hi q][hj q]
    float *hi = sc + qq;
    float *hj = hi + q;
    const float fq = (float)q;
    for (uint64_t p = (uint64_t)blockIdx.x * wpb + warp; p < npairs; p += (uint64_t)gridDim.x * wpb) {
        const float *Jb = J + p * qq;
        float *dJb = dJ + p * qq;
        // row sums
        for (uint32_t li = lane; li < qq; li += 32) sc[li] = Jb[li] + dJb[li];
        __syncwarp();
        rows_tree(sc, q, lane);
        for (uint32_t a = lane; a < q; a += 32) hi[a] = sc[q * a] / fq;
        __syncwarp();
        // column sums (transpose into scratch)
        for (uint32_t li = lane; li < qq; li += 32) sc[q * (li % q) + li / q] = Jb[li] + dJb[li];
        __syncwarp();
        rows_tree(sc, q, lane);
        for (uint32_t b = lane; b < q; b += 32) hj[b] = sc[q * b] / fq;
        __syncwarp();
        // total of the column sums
        uint32_t m = q;
        while (m > 1) {
            uint32_t odd = m & 1;
            m = (m + 1) >> 1;
            for (uint32_t li = lane; li < m - odd; li += 32) sc[q * li] = sc[q * li] + sc[q * (li + m)];
            __syncwarp();
        }
        float mean = sc[0] / fq / fq;
        __syncwarp();
        for (uint32_t a = lane; a < q; a += 32) {
            hi[a] = hi[a] - mean;
            hj[a] = hj[a] - mean;
        }
        __syncwarp();
        for (uint32_t li = lane; li < qq; li += 32) {
            float Jp = dJb[li];
            float Jt0 = Jb[li] + Jp;
            float J0 = Jt0 - (hi[li / q] + hj[li % q]) - mean;
            float R;
            if (L2) R = -lJ * J0 * gamma / (bi[p * qq + li] + pc);
            else R = -lJ * ocl_sign(J0) * gamma / (bi[p * qq + li] + pc);
            if (ocl_sign(J0) != ocl_sign(J0 + R)) Jp = Jp - J0;
            else Jp = Jp + R;
            dJb[li] = Jp;
        }
        __syncwarp();
    }
}

// reg_l1z / reg_l2z for q*q <= 512 with the trees run per lane.  The
// reference's zeroGauge (mcmc.cl:764-822) sums each row and each column of
// the block with the same odd-aware tree (level m -> (m+1)/2: element b
// gets b + m' for b < m' - odd) and the column sums with that tree again.
// Here lane a owns row a (and, in a transposed copy, column a) and runs its
// tree sequentially, level by level -- the same additions of the same
// operands, so the sums are bit-identical -- instead of every level looping
// over all q*q cells with an index modulo.  The block's values and dJ stay
// in registers for the final pass.
__device__ __forceinline__ void tree_level(float *__restrict__ w, const float *__restrict__ rd, uint32_t cnt,
                                           uint32_t stride) {
    // w[b] += rd[b] for b < cnt: the read half (from element m on) and the
    // written half (below m) do not overlap, so the adds of a level are
    // independent
#pragma unroll 4
    for (uint32_t b = 0; b < cnt; ++b) w[b * stride] = w[b * stride] + rd[b * stride];
}

__device__ __forceinline__ float lane_tree(float *r, uint32_t q, uint32_t stride) {
    uint32_t m = q;
    while (m > 1) {
        const uint32_t odd = m & 1;
        m = (m + 1) >> 1;
        tree_level(r, r + m * stride, m - odd, stride);
    }
    return r[0];
}

// PER: cells per lane, ceil(q*q / 32) rounded up to a power of two.
template <bool L2, uint32_t PER>
__global__ void __launch_bounds__(256) k_reg_lz_rows(const float *__restrict__ bi, float gamma, float pc, float lJ,
                                                     const float *__restrict__ J, float *__restrict__ dJ,
                                                     uint64_t npairs, uint32_t q) {
    extern __shared__ float sm[];
    const uint32_t qq = q * q;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t wpb = blockDim.x >> 5;
    const uint32_t WS = 2 * qq + 2 * q + 1;
    float *xs = sm + warp * WS;  // [q*q] rows
    float *xt = xs + qq;         // [q*q] columns (transposed)
    float *hi = xt + qq;
    float *hj = hi + q;
    float *mean_s = hj + q;
    const float fq = (float)q;
    // this lane's cells li = lane + 32 k, as (a, b) with li = a q + b
    const uint32_t a0 = lane / q, b0 = lane - a0 * q, da = 32 / q, db = 32 - da * q;
    for (uint64_t p = (uint64_t)blockIdx.x * wpb + warp; p < npairs; p += (uint64_t)gridDim.x * wpb) {
        const float *Jb = J + p * qq;
        float *dJb = dJ + p * qq;
        const float *bb = bi + p * qq;
        float xv[PER], dv[PER], bv[PER];
        // every global load of the block first (all in flight together),
        // then the shared-memory copies
#pragma unroll
        for (uint32_t k = 0; k < PER; ++k) {
            const uint32_t li = lane + 32 * k;
            if (li < qq) {
                dv[k] = dJb[li];
                xv[k] = Jb[li];
                bv[k] = bb[li];
            }
        }
        uint32_t a = a0, b = b0;
#pragma unroll
        for (uint32_t k = 0; k < PER; ++k) {
            const uint32_t li = lane + 32 * k;
            if (li < qq) {
                xv[k] = xv[k] + dv[k];
                xs[li] = xv[k];
                xt[b * q + a] = xv[k];
            }
            b += db;
            a += da;
            if (b >= q) {
                b -= q;
                ++a;
            }
        }
        __syncwarp();
        if (lane < q) {
            hi[lane] = lane_tree(xs + lane * q, q, 1) / fq;
            hj[lane] = lane_tree(xt + lane * q, q, 1) / fq;  // xt[lane*q] keeps column lane's sum
        }
        __syncwarp();
        if (lane == 0) *mean_s = lane_tree(xt, q, q) / fq / fq;  // total of the column sums
        __syncwarp();
        const float mean = *mean_s;
        if (lane < q) {
            hi[lane] = hi[lane] - mean;
            hj[lane] = hj[lane] - mean;
        }
        __syncwarp();
        a = a0;
        b = b0;
#pragma unroll
        for (uint32_t k = 0; k < PER; ++k) {
            const uint32_t li = lane + 32 * k;
            if (li < qq) {
                const float J0 = xv[k] - (hi[a] + hj[b]) - mean;
                float R;
                if (L2) R = -lJ * J0 * gamma / (bv[k] + pc);
                else R = -lJ * ocl_sign(J0) * gamma / (bv[k] + pc);
                float Jp = dv[k];
                if (ocl_sign(J0) != ocl_sign(J0 + R)) Jp = Jp - J0;
                else Jp = Jp + R;
                dJb[li] = Jp;
            }
            b += db;
            a += da;
            if (b >= q) {
                b -= q;
                ++a;
            }
        }
        __syncwarp();
    }
}

// reg_l1z / reg_l2z with q known at compile time: lane a holds row a and
// column a of the block in registers and runs the odd-aware tree of
// zeroGauge on them (level m -> (m+1)/2: element b gets b + m' for
// b < m' - odd), fully unrolled -- the same additions of the same operands
// as k_reg_lz / k_reg_lz_rows, so the sums are bit-identical; the mean is
// the same tree over the column sums, gathered by shuffles.  The block
// (J + dJ) and dJ are staged in shared memory by coalesced loads.
template <uint32_t Q>
__device__ __forceinline__ float tree_reg(float (&w)[Q]) {
    uint32_t m = Q;
#pragma unroll
    for (int lev = 0; lev < 8; ++lev) {
        if (m > 1) {
            const uint32_t odd = m & 1;
            m = (m + 1) >> 1;
#pragma unroll
            for (uint32_t b = 0; b < Q; ++b)
                if (b + odd < m && b + m < Q) w[b] = w[b] + w[b + m];
        }
    }
    return w[0];
}

template <bool L2, uint32_t Q>
__global__ void __launch_bounds__(256) k_reg_lz_q(const float *__restrict__ bi, float gamma, float pc, float lJ,
                                                  const float *__restrict__ J, float *__restrict__ dJ,
                                                  uint64_t npairs) {
    constexpr uint32_t QQ = Q * Q, PER = (QQ + 31) / 32;
    __shared__ float xs[8][QQ + 1], ds[8][QQ + 1];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const float fq = (float)Q;
    float *x = xs[warp], *d = ds[warp];
    for (uint64_t p = (uint64_t)blockIdx.x * 8 + warp; p < npairs; p += (uint64_t)gridDim.x * 8) {
        const float *Jb = J + p * QQ;
        float *dJb = dJ + p * QQ;
        const float *bb = bi + p * QQ;
        float jv[PER], dv[PER];
#pragma unroll
        for (uint32_t k = 0; k < PER; ++k) {
            const uint32_t li = lane + 32 * k;
            if (li < QQ) {
                dv[k] = dJb[li];
                jv[k] = Jb[li];
            }
        }
#pragma unroll
        for (uint32_t k = 0; k < PER; ++k) {
            const uint32_t li = lane + 32 * k;
            if (li < QQ) {
                x[li] = jv[k] + dv[k];
                d[li] = dv[k];
            }
        }
        __syncwarp();
        float rsum = 0.0f, csum = 0.0f;
        if (lane < Q) {
            float w[Q];
#pragma unroll
            for (uint32_t b = 0; b < Q; ++b) w[b] = x[lane * Q + b];
            rsum = tree_reg<Q>(w);
#pragma unroll
            for (uint32_t a = 0; a < Q; ++a) w[a] = x[a * Q + lane];
            csum = tree_reg<Q>(w);
        }
        float cs[Q];
#pragma unroll
        for (uint32_t b = 0; b < Q; ++b) cs[b] = __shfl_sync(0xffffffffu, csum, b);
        const float mean = tree_reg<Q>(cs) / fq / fq;
        const float hi = rsum / fq - mean, hj = csum / fq - mean;
#pragma unroll
        for (uint32_t k = 0; k < PER; ++k) {
            const uint32_t li = lane + 32 * k;
            const uint32_t lc = li < QQ ? li : QQ - 1;
            const uint32_t a = lc / Q, b = lc - a * Q;
            const float ha = __shfl_sync(0xffffffffu, hi, a), hb = __shfl_sync(0xffffffffu, hj, b);
            if (li < QQ) {
                const float J0 = x[li] - (ha + hb) - mean;
                const float bv = bb[li];
                float R;
                if (L2) R = -lJ * J0 * gamma / (bv + pc);
                else R = -lJ * ocl_sign(J0) * gamma / (bv + pc);
                float Jp = d[li];
                if (ocl_sign(J0) != ocl_sign(J0 + R)) Jp = Jp - J0;
                else Jp = Jp + R;
                dJb[li] = Jp;
            }
        }
        __syncwarp();
    }
}

// ------------------------------------------------------------ reductions
// Workspace: [ticket counter (uint32, padded to 16 B)][partials: NBLK x 4 doubles]
constexpr uint32_t RED_BLOCKS = 296;
constexpr uint32_t RED_THREADS = 512;

enum RedMode : uint32_t { RM_WEIGHTS = 1, RM_MIN = 2, RM_STATS = 4 };

struct RedOut {
    float *weights;   // RM_WEIGHTS: output
    float *minout;    // RM_MIN
    float *stats;     // RM_STATS: {sum, sum2} float
    double *stats64;  // RM_STATS: {sum, sum2} double (nullable)
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_min_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

// in = dE when RM_WEIGHTS (weights computed as exp(-dE + ref)), else weights.
__global__ void __launch_bounds__(RED_THREADS) k_reduce(const float *__restrict__ in, uint32_t n,
                                                        float ref_host, const float *ref_dev, uint32_t mode,
                                                        RedOut o, unsigned char *ws) {
    const float ref = ref_dev ? *ref_dev : ref_host;
    unsigned int *ticket = reinterpret_cast<unsigned int *>(ws);
    double *part = reinterpret_cast<double *>(ws + 16);
    __shared__ double s_sum[RED_THREADS / 32], s_sum2[RED_THREADS / 32], s_mind[RED_THREADS / 32];
    __shared__ float s_min[RED_THREADS / 32];
    __shared__ bool s_last;
    double a = 0.0, b = 0.0;
    float mn = 0.0f;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        float v = in[k];
        if (mode & RM_MIN) mn = fminf(v, mn);
        if (mode & RM_WEIGHTS) {
            v = expf(-v + ref);
            o.weights[k] = v;
        }
        if (mode & RM_STATS) {
            double dv = (double)v;
            a += dv;
            b += dv * dv;
        }
    }
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    a = warp_sum(a);
    b = warp_sum(b);
    mn = warp_min(mn);
    if (lane == 0) {
        s_sum[warp] = a;
        s_sum2[warp] = b;
        s_min[warp] = mn;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ta = 0.0, tb = 0.0;
        float tm = 0.0f;
        for (uint32_t w = 0; w < blockDim.x / 32; ++w) {
            ta += s_sum[w];
            tb += s_sum2[w];
            tm = fminf(tm, s_min[w]);
        }
        part[4 * blockIdx.x + 0] = ta;
        part[4 * blockIdx.x + 1] = tb;
        part[4 * blockIdx.x + 2] = (double)tm;
        __threadfence();
        unsigned int t = atomicAdd(ticket, 1u);
        s_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    // the last CTA combines the partials: every thread loads its share from
    // L2 (ld.global.cg: written by other CTAs, ordered by their fences and
    // the ticket), then warp shuffles and a fixed pass over the warps -- a
    // fixed order, so the sums are deterministic
    if (s_last) {
        __threadfence();
        double ta = 0.0, tb = 0.0, tm = 0.0;
        for (uint32_t k = threadIdx.x; k < gridDim.x; k += blockDim.x) {
            ta += __ldcg(&part[4 * k + 0]);
            tb += __ldcg(&part[4 * k + 1]);
            tm = fmin(tm, __ldcg(&part[4 * k + 2]));
        }
        ta = warp_sum(ta);
        tb = warp_sum(tb);
        tm = warp_min_d(tm);
        if (lane == 0) {
            s_sum[warp] = ta;
            s_sum2[warp] = tb;
            s_mind[warp] = tm;
        }
        __syncthreads();
        if (threadIdx.x != 0) return;
        ta = 0.0, tb = 0.0, tm = 0.0;
        for (uint32_t w = 0; w < blockDim.x / 32; ++w) {
            ta += s_sum[w];
            tb += s_sum2[w];
            tm = fmin(tm, s_mind[w]);
        }
        if (mode & RM_STATS) {
            o.stats[0] = (float)ta;
            o.stats[1] = (float)tb;
            if (o.stats64) {
                o.stats64[0] = ta;
                o.stats64[1] = tb;
            }
        }
        if (mode & RM_MIN) *o.minout = (float)tm;
        *ticket = 0u;  // ready for the next call
    }
}

// min(0, min data): per-CTA minimum, then an integer atomicMax on the bit
// pattern -- for non-positive floats a larger magnitude is a larger unsigned
// pattern, so the result is exact and order independent.
__global__ void __launch_bounds__(RED_THREADS) k_min(const float *__restrict__ in, uint32_t n,
                                                     unsigned int *out) {
    __shared__ float s_min[RED_THREADS / 32];
    float mn = 0.0f;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        mn = fminf(in[k], mn);
    mn = warp_min(mn);
    if ((threadIdx.x & 31) == 0) s_min[threadIdx.x >> 5] = mn;
    __syncthreads();
    if (threadIdx.x == 0) {
        float tm = 0.0f;
        for (uint32_t w = 0; w < blockDim.x / 32; ++w) tm = fminf(tm, s_min[w]);
        if (tm < 0.0f) atomicMax(out, __float_as_uint(tm));
    }
}

__global__ void k_dE_to_weights(float ref, const float *__restrict__ dE, float *w, uint32_t n) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) w[k] = expf(-dE[k] + ref);
}

__global__ void k_fixed_beta(float beta, float ref, const float *__restrict__ E, float *w, uint32_t n) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) w[k] = expf((beta - 1.0f) * (E[k] - ref));
}

__global__ void k_add(float *dst, const float *__restrict__ src, uint32_t n) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) dst[k] += src[k];
}

static size_t red_ws_bytes() { return 16 + (size_t)RED_BLOCKS * 4 * sizeof(double); }

static int launch_reduce(const float *in, uint32_t n, float ref, uint32_t mode, RedOut o, void *ws,
                         size_t ws_bytes, cudaStream_t st, const char *what, const float *ref_dev = nullptr) {
    if (ws_bytes < red_ws_bytes()) return fail(MI3_ERR_WORKSPACE, std::string(what) + ": workspace too small");
    if (!aligned(ws, 16)) return fail(MI3_ERR_ALIGN, std::string(what) + ": workspace alignment");
    uint32_t blocks = std::min<uint32_t>(RED_BLOCKS, std::max<uint32_t>(1, (n + RED_THREADS - 1) / RED_THREADS));
    if (cudaMemsetAsync(ws, 0, 16, st) != cudaSuccess) return check_launch(what);
    k_reduce<<<blocks, RED_THREADS, 0, st>>>(in, n, ref, ref_dev, mode, o, reinterpret_cast<unsigned char *>(ws));
    return check_launch(what);
}

}  // namespace mi3

using namespace mi3;

extern "C" int mi3_update_j(const float *bi_target, const float *bi, float gamma, float pc, const float *Ji,
                            float *Jo, uint32_t L, uint32_t q, void *stream) {
    if (!bi_target || !bi || !Ji || !Jo) return fail(MI3_ERR_ARG, "mi3_update_j: null pointer");
    if (L < 2 || q < 1) return fail(MI3_ERR_ARG, "mi3_update_j: bad L/q");
    uint64_t n = npairs_of(L) * q * q;
    k_update_j<<<(uint32_t)((n + 255) / 256), 256, 0, as_stream(stream)>>>(bi_target, bi, gamma, pc, Ji, Jo, n);
    return check_launch("mi3_update_j");
}

static int reg_lz(bool l2, const float *bi, float gamma, float pc, float lJ, const float *J, float *dJ,
                  uint32_t L, uint32_t q, void *stream) {
    const char *name = l2 ? "mi3_reg_l2z" : "mi3_reg_l1z";
    if (!bi || !J || !dJ) return fail(MI3_ERR_ARG, std::string(name) + ": null pointer");
    if (L < 2 || q < 1 || q * q > 4096) return fail(MI3_ERR_ARG, std::string(name) + ": bad L/q");
    uint64_t np = npairs_of(L);
    uint32_t tb = 256;
    if (q == 21 || q == 4) {  // the protein and nucleotide alphabets, q fixed at compile time
        using K = void (*)(const float *, float, float, float, const float *, float *, uint64_t);
        K k;
        if (q == 21) k = l2 ? (K)k_reg_lz_q<true, 21> : (K)k_reg_lz_q<false, 21>;
        else k = l2 ? (K)k_reg_lz_q<true, 4> : (K)k_reg_lz_q<false, 4>;
        const uint32_t grid = (uint32_t)std::min<uint64_t>((np + 7) / 8, 148 * 32);
        k<<<grid, tb, 0, as_stream(stream)>>>(bi, gamma, pc, lJ, J, dJ, np);
        return check_launch(name);
    }
    if (q * q <= 512) {  // up to 16 cells per lane (q <= 22); larger blocks use the generic kernel
        using K = void (*)(const float *, float, float, float, const float *, float *, uint64_t, uint32_t);
        const uint32_t per = (q * q + 31) / 32;
        K k = nullptr;
        if (per <= 2) k = l2 ? (K)k_reg_lz_rows<true, 2> : (K)k_reg_lz_rows<false, 2>;
        else if (per <= 4) k = l2 ? (K)k_reg_lz_rows<true, 4> : (K)k_reg_lz_rows<false, 4>;
        else if (per <= 8) k = l2 ? (K)k_reg_lz_rows<true, 8> : (K)k_reg_lz_rows<false, 8>;
        else k = l2 ? (K)k_reg_lz_rows<true, 16> : (K)k_reg_lz_rows<false, 16>;
        const size_t sm2 = (size_t)(tb / 32) * (2 * q * q + 2 * q + 1) * 4;
        const uint32_t grid2 = (uint32_t)std::min<uint64_t>((np + 7) / 8, 148 * 16);
        if (sm2 > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2);
        k<<<grid2, tb, sm2, as_stream(stream)>>>(bi, gamma, pc, lJ, J, dJ, np, q);
        return check_launch(name);
    }
    size_t smem = (size_t)(tb / 32) * (q * q + 2 * q + 2) * 4;
    uint32_t grid = (uint32_t)std::min<uint64_t>((np + 7) / 8, 148 * 16);
    if (smem > 48 * 1024) {
        if (l2) cudaFuncSetAttribute(k_reg_lz<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        else cudaFuncSetAttribute(k_reg_lz<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    }
    if (l2) k_reg_lz<true><<<grid, tb, smem, as_stream(stream)>>>(bi, gamma, pc, lJ, J, dJ, np, q);
    else k_reg_lz<false><<<grid, tb, smem, as_stream(stream)>>>(bi, gamma, pc, lJ, J, dJ, np, q);
    return check_launch(name);
}

extern "C" int mi3_reg_l1z(const float *bi, float gamma, float pc, float lJ, const float *J, float *dJ,
                           uint32_t L, uint32_t q, void *stream) {
    return reg_lz(false, bi, gamma, pc, lJ, J, dJ, L, q, stream);
}

extern "C" int mi3_reg_l2z(const float *bi, float gamma, float pc, float lJ, const float *J, float *dJ,
                           uint32_t L, uint32_t q, void *stream) {
    return reg_lz(true, bi, gamma, pc, lJ, J, dJ, L, q, stream);
}

extern "C" size_t mi3_weight_stats_workspace(uint32_t n) {
    (void)n;
    return red_ws_bytes();
}

extern "C" int mi3_min_floats(const float *data, uint32_t len, float *out, void *stream) {
    if (!data || !out) return fail(MI3_ERR_ARG, "mi3_min_floats: null pointer");
    cudaStream_t st = as_stream(stream);
    if (cudaMemsetAsync(out, 0, sizeof(float), st) != cudaSuccess) return check_launch("mi3_min_floats: memset");
    if (len == 0) return MI3_OK;
    uint32_t blocks = std::min<uint32_t>(RED_BLOCKS, (len + RED_THREADS - 1) / RED_THREADS);
    k_min<<<blocks, RED_THREADS, 0, st>>>(data, len, reinterpret_cast<unsigned int *>(out));
    return check_launch("mi3_min_floats");
}

extern "C" int mi3_dE_to_weights(float ref_E, const float *dE, float *weights, uint32_t n, void *stream) {
    if (!dE || !weights) return fail(MI3_ERR_ARG, "mi3_dE_to_weights: null pointer");
    if (n == 0) return MI3_OK;
    k_dE_to_weights<<<(n + 255) / 256, 256, 0, as_stream(stream)>>>(ref_E, dE, weights, n);
    return check_launch("mi3_dE_to_weights");
}

extern "C" int mi3_fixed_beta_weights(float beta, float ref_E, const float *E, float *weights, uint32_t n,
                                      void *stream) {
    if (!E || !weights) return fail(MI3_ERR_ARG, "mi3_fixed_beta_weights: null pointer");
    if (n == 0) return MI3_OK;
    k_fixed_beta<<<(n + 255) / 256, 256, 0, as_stream(stream)>>>(beta, ref_E, E, weights, n);
    return check_launch("mi3_fixed_beta_weights");
}

extern "C" int mi3_weight_stats(const float *weights, uint32_t n, float *out2, double *out2_f64,
                                void *workspace, size_t ws_bytes, void *stream) {
    if (!weights || !out2 || !workspace) return fail(MI3_ERR_ARG, "mi3_weight_stats: null pointer");
    RedOut o{nullptr, nullptr, out2, out2_f64};
    return launch_reduce(weights, n, 0.0f, RM_STATS, o, workspace, ws_bytes, as_stream(stream),
                         "mi3_weight_stats");
}

extern "C" int mi3_weights_fused(float ref_E, const float *dE, float *weights, uint32_t n, float *minout,
                                 float *out2, double *out2_f64, void *workspace, size_t ws_bytes,
                                 void *stream) {
    if (!dE || !weights || !minout || !out2 || !workspace)
        return fail(MI3_ERR_ARG, "mi3_weights_fused: null pointer");
    RedOut o{weights, minout, out2, out2_f64};
    return launch_reduce(dE, n, ref_E, RM_WEIGHTS | RM_MIN | RM_STATS, o, workspace, ws_bytes,
                         as_stream(stream), "mi3_weights_fused");
}

extern "C" int mi3_weights_fused_dev(const float *ref_dev, const float *dE, float *weights, uint32_t n,
                                     float *minout, float *out2, double *out2_f64, void *workspace,
                                     size_t ws_bytes, void *stream) {
    if (!ref_dev || !dE || !weights || !minout || !out2 || !workspace)
        return fail(MI3_ERR_ARG, "mi3_weights_fused_dev: null pointer");
    if (ref_dev == minout) return fail(MI3_ERR_ARG, "mi3_weights_fused_dev: ref_dev must not alias minout");
    RedOut o{weights, minout, out2, out2_f64};
    return launch_reduce(dE, n, 0.0f, RM_WEIGHTS | RM_MIN | RM_STATS, o, workspace, ws_bytes, as_stream(stream),
                         "mi3_weights_fused_dev", ref_dev);
}

extern "C" int mi3_add_float_bufs(float *dst, const float *src, uint32_t n, void *stream) {
    if (!dst || !src) return fail(MI3_ERR_ARG, "mi3_add_float_bufs: null pointer");
    if (n == 0) return MI3_OK;
    k_add<<<(n + 255) / 256, 256, 0, as_stream(stream)>>>(dst, src, n);
    return check_launch("mi3_add_float_bufs");
}
