// roundstats.cu -- per-round host work of the quasi-Newton loop done on the
// device in FP64: the fieldless-even gauge transform of the couplings and the
// bimarginal error statistics (SSR, relative error, max deviation, X).
//
// The reference does both on the host in numpy float64 / float32 every round
// (changeGauge.py:37-155 fieldlessGaugeEven; NewtonSteps.py:33-54
// bimarg_stats and printstats), which means reading the 26796 x 441 coupling
// and bimarginal tables back from the device and sending J down again.  Here
// J stays resident.  All reductions have a fixed thread-to-element
// assignment and a fixed tree order, so results are deterministic.
#include "tiling.cuh"

namespace mi3 {


// Per pair: column means m1[b] = mean_a J(a,b), row means m2[a] = mean_b
// J(a,b) and the pair mean mJ = mean_b m1[b] (changeGauge.py:79-81).
__global__ void k_gauge_means(const float *__restrict__ J, double *m1, double *m2, double *mJ, uint32_t q) {
    const uint32_t p = blockIdx.x;
    const float *Jp = J + (size_t)p * q * q;
    const double invq = 1.0 / (double)q;
    for (uint32_t t = threadIdx.x; t < q; t += blockDim.x) {
        double c = 0.0, r = 0.0;
        for (uint32_t k = 0; k < q; ++k) {
            c += (double)Jp[k * q + t];
            r += (double)Jp[t * q + k];
        }
        m1[(size_t)p * q + t] = c * invq;
        m2[(size_t)p * q + t] = r * invq;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (uint32_t b = 0; b < q; ++b) s += m1[(size_t)p * q + b];
        mJ[p] = s * invq;
    }
}

// The same, one warp per pair and 8 pairs per CTA (q <= 32): lane t holds
// column t and row t, summed in the same order; the pair mean adds the
// column means in order b = 0..q-1 (shuffles), as above.
__global__ void __launch_bounds__(256) k_gauge_means_w(const float *__restrict__ J, double *m1, double *m2,
                                                       double *mJ, uint32_t q, uint32_t np) {
    __shared__ float tile[8][32 * 32];
    const uint32_t w = threadIdx.x >> 5, t = threadIdx.x & 31;
    const uint32_t p = blockIdx.x * 8 + w;
    if (p >= np) return;  // the whole warp
    const uint32_t qq = q * q;
    const float *Jp = J + (size_t)p * qq;
    float *Js = tile[w];
    for (uint32_t e = t; e < qq; e += 32) Js[e] = Jp[e];  // coalesced, all in flight
    __syncwarp();
    const double invq = 1.0 / (double)q;
    double c = 0.0, r = 0.0;
    if (t < q) {
        for (uint32_t k = 0; k < q; ++k) {
            c += (double)Js[k * q + t];
            r += (double)Js[t * q + k];
        }
        m1[(size_t)p * q + t] = c * invq;
        m2[(size_t)p * q + t] = r * invq;
    }
    double s = 0.0;
    for (uint32_t b = 0; b < q; ++b) s += __shfl_sync(0xffffffffu, c * invq, b);
    if (t == 0) mJ[p] = s * invq;
}

// Per site k: the zero-gauge field divided by L-1.  zeroJGauge gives
// h_k(c) = -sum(mJ)/L + sum_{i<k} m1[(i,k)][c] + sum_{j>k} m2[(k,j)][c]
// (changeGauge.py:86-90), and zeroGauge subtracts its mean over c; the mean
// of m1 and of m2 over c is mJ, so the centred field is
// sum_{i<k} (m1[(i,k)][c] - mJ) + sum_{j>k} (m2[(k,j)][c] - mJ).
__global__ void k_gauge_fields(const double *__restrict__ m1, const double *__restrict__ m2,
                               const double *__restrict__ mJ, double *hd, uint32_t L, uint32_t q) {
    const uint32_t k = blockIdx.x;
    for (uint32_t c = threadIdx.x; c < q; c += blockDim.x) {
        double h = 0.0;
        for (uint32_t i = 0; i < k; ++i) {
            uint64_t p = pair_index(i, k, L);
            h += m1[p * q + c] - mJ[p];
        }
        for (uint32_t j = k + 1; j < L; ++j) {
            uint64_t p = pair_index(k, j, L);
            h += m2[p * q + c] - mJ[p];
        }
        hd[(size_t)k * q + c] = h / (double)(L - 1);
    }
}

// The same with 8 warps per site (q <= 32): warp w sums its contiguous
// share of the site's L-1 pairs (in pair order), lane c its field entry;
// the eight partial sums are added in warp order.
__global__ void __launch_bounds__(256) k_gauge_fields_w(const double *__restrict__ m1, const double *__restrict__ m2,
                                                        const double *__restrict__ mJ, double *hd, uint32_t L,
                                                        uint32_t q) {
    __shared__ double part[8][32];
    const uint32_t k = blockIdx.x, w = threadIdx.x >> 5, c = threadIdx.x & 31;
    const uint32_t n = L - 1, chunk = (n + 7) / 8;
    const uint32_t e0 = min(n, w * chunk), e1 = min(n, e0 + chunk);
    double h = 0.0;
    if (c < q) {
#pragma unroll 4
        for (uint32_t e = e0; e < e1; ++e) {
            // entries e < k are the pairs (e, k), the others (k, e + 1)
            if (e < k) {
                const uint64_t p = pair_index(e, k, L);
                h += m1[p * q + c] - mJ[p];
            } else {
                const uint64_t p = pair_index(k, e + 1, L);
                h += m2[p * q + c] - mJ[p];
            }
        }
    }
    part[w][c] = h;
    __syncthreads();
    if (w == 0 && c < q) {
        double s = part[0][c];
        for (uint32_t x = 1; x < 8; ++x) s += part[x][c];
        hd[(size_t)k * q + c] = s / (double)(L - 1);
    }
}

// Pair p -> (i, j), i < j, in closed form: row i starts at i (2L - i - 1) / 2.
__device__ __forceinline__ void pair_decode_fast(uint32_t p, uint32_t L, uint32_t &i, uint32_t &j) {
    const double b = 2.0 * (double)L - 1.0;
    int64_t r = (int64_t)floor((b - sqrt(b * b - 8.0 * (double)p)) * 0.5);
    auto start = [&](int64_t x) { return x * (2 * (int64_t)L - x - 1) / 2; };
    if (r < 0) r = 0;
    while (r + 1 < (int64_t)L && start(r + 1) <= (int64_t)p) ++r;
    while (r > 0 && start(r) > (int64_t)p) --r;
    i = (uint32_t)r;
    j = (uint32_t)(r + 1 + ((int64_t)p - start(r)));
}

// k_gauge_apply with one warp per pair, 8 pairs per CTA.
__global__ void __launch_bounds__(256) k_gauge_apply_w(const float *J, float *Jout, const double *__restrict__ m1,
                                                       const double *__restrict__ m2, const double *__restrict__ mJ,
                                                       const double *__restrict__ hd, uint32_t L, uint32_t q,
                                                       uint32_t np) {
    const uint32_t p = blockIdx.x * 8 + (threadIdx.x >> 5), l = threadIdx.x & 31;
    if (p >= np) return;
    uint32_t i, j;
    pair_decode_fast(p, L, i, j);
    const uint32_t qq = q * q;
    const float *Jp = J + (size_t)p * qq;
    float *Op = Jout + (size_t)p * qq;
    const double mj = mJ[p];
    for (uint32_t e = l; e < qq; e += 32) {
        const uint32_t a = e / q, b = e - a * q;
        double v = (double)Jp[e] - m1[(size_t)p * q + b] - m2[(size_t)p * q + a] + mj;
        v = v + hd[(size_t)i * q + a] + hd[(size_t)j * q + b];
        Op[e] = (float)v;
    }
}

// J0 = J - m1[b] - m2[a] + mJ, then the fields folded evenly into the L-1
// couplings of each site: J0 + hd_i[a] + hd_j[b] (changeGauge.py:79-82,
// 116-135); rounded to float once at the end.
__global__ void k_gauge_apply(const float *J, float *Jout, const double *__restrict__ m1,
                              const double *__restrict__ m2, const double *__restrict__ mJ,
                              const double *__restrict__ hd, uint32_t L, uint32_t q) {
    const uint32_t p = blockIdx.x;
    uint32_t i, j;
    pair_decode_fast(p, L, i, j);
    const uint32_t qq = q * q;
    const float *Jp = J + (size_t)p * qq;
    float *Op = Jout + (size_t)p * qq;
    for (uint32_t e = threadIdx.x; e < qq; e += blockDim.x) {
        uint32_t a = e / q, b = e - a * q;
        double v = (double)Jp[e] - m1[(size_t)p * q + b] - m2[(size_t)p * q + a] + mJ[p];
        v = v + hd[(size_t)i * q + a] + hd[(size_t)j * q + b];
        Op[e] = (float)v;
    }
}

// ------------------------------------------------------------ statistics
// Per pair six partials: SSR, max |t-m|, sum of |t-m|/t over t > 0.01, the
// number of such entries, X_model = sum J (m - m_a m_b), X_target likewise
// with t (NewtonSteps.py:33-54; m_a, m_b are the pair's own row and column
// sums, indepF in potts_common.py).
constexpr int STAT_THREADS = 128;
constexpr int NSTAT = 6;

__device__ __forceinline__ double block_sum(double v, double *red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += red[k];
    return s;  // valid in thread 0
}

__device__ __forceinline__ double block_max(double v, double *red) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s = fmax(s, red[k]);
    return s;
}

__global__ void __launch_bounds__(STAT_THREADS) k_pair_stats(const float *__restrict__ tgt,
                                                             const float *__restrict__ mdl,
                                                             const float *__restrict__ J, double *part,
                                                             uint32_t q) {
    extern __shared__ double sh[];  // rows/cols sums of model and target: 4*q doubles
    __shared__ double red[STAT_THREADS / 32];
    double *ma = sh, *mb = sh + q, *ta = sh + 2 * q, *tb = sh + 3 * q;
    const uint32_t p = blockIdx.x, qq = q * q;
    const float *T = tgt + (size_t)p * qq, *M = mdl + (size_t)p * qq;
    for (uint32_t t = threadIdx.x; t < q; t += blockDim.x) {
        double sm_r = 0, sm_c = 0, st_r = 0, st_c = 0;
        for (uint32_t k = 0; k < q; ++k) {
            sm_r += M[t * q + k];
            sm_c += M[k * q + t];
            st_r += T[t * q + k];
            st_c += T[k * q + t];
        }
        ma[t] = sm_r; mb[t] = sm_c; ta[t] = st_r; tb[t] = st_c;
    }
    __syncthreads();
    double ssr = 0, mx = 0, rel = 0, cnt = 0, xm = 0, xt = 0;
    for (uint32_t e = threadIdx.x; e < qq; e += blockDim.x) {
        const double t = T[e], m = M[e], d = t - m;
        ssr += d * d;
        mx = fmax(mx, fabs(d));
        if (T[e] > 0.01f) {
            rel += fabs(d) / t;
            cnt += 1.0;
        }
        if (J) {
            const uint32_t a = e / q, b = e - a * q;
            const double jv = J[(size_t)p * qq + e];
            xm += jv * (m - ma[a] * mb[b]);
            xt += jv * (t - ta[a] * tb[b]);
        }
    }
    double r0 = block_sum(ssr, red);
    double r1 = block_max(mx, red);
    double r2 = block_sum(rel, red);
    double r3 = block_sum(cnt, red);
    double r4 = block_sum(xm, red);
    double r5 = block_sum(xt, red);
    if (threadIdx.x == 0) {
        double *o = part + (size_t)p * NSTAT;
        o[0] = r0; o[1] = r1; o[2] = r2; o[3] = r3; o[4] = r4; o[5] = r5;
    }
}

// The same, one warp per pair and 8 pairs per CTA (q <= 32): lanes hold the
// row and column sums (same order), elements e = lane + 32 k, then a
// shuffle tree per statistic.
__global__ void __launch_bounds__(256) k_pair_stats_w(const float *__restrict__ tgt, const float *__restrict__ mdl,
                                                      const float *__restrict__ J, double *part, uint32_t q,
                                                      uint32_t np) {
    __shared__ double sums[8][4][32];
    extern __shared__ float stage[];  // [8 warps][2][q q]: the pair's target and model
    const uint32_t w = threadIdx.x >> 5, l = threadIdx.x & 31;
    const uint32_t p = blockIdx.x * 8 + w;
    if (p >= np) return;  // the whole warp
    const uint32_t qq = q * q;
    const float *Tg = tgt + (size_t)p * qq, *Mg = mdl + (size_t)p * qq;
    float *T = stage + (size_t)w * 2 * qq, *M = T + qq;
    for (uint32_t e = l; e < qq; e += 32) {  // coalesced, all in flight
        T[e] = Tg[e];
        M[e] = Mg[e];
    }
    __syncwarp();
    double *ma = sums[w][0], *mb = sums[w][1], *ta = sums[w][2], *tb = sums[w][3];
    if (J && l < q) {
        double sm_r = 0, sm_c = 0, st_r = 0, st_c = 0;
        for (uint32_t k = 0; k < q; ++k) {
            sm_r += M[l * q + k];
            sm_c += M[k * q + l];
            st_r += T[l * q + k];
            st_c += T[k * q + l];
        }
        ma[l] = sm_r; mb[l] = sm_c; ta[l] = st_r; tb[l] = st_c;
    }
    __syncwarp();
    double v[NSTAT] = {0, 0, 0, 0, 0, 0};
    for (uint32_t e = l; e < qq; e += 32) {
        const double t = T[e], m = M[e], d = t - m;
        v[0] += d * d;
        v[1] = fmax(v[1], fabs(d));
        if (T[e] > 0.01f) {
            v[2] += fabs(d) / t;
            v[3] += 1.0;
        }
        if (J) {
            const uint32_t a = e / q, b = e - a * q;
            const double jv = J[(size_t)p * qq + e];
            v[4] += jv * (m - ma[a] * mb[b]);
            v[5] += jv * (t - ta[a] * tb[b]);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int k = 0; k < NSTAT; ++k) {
            const double x = __shfl_down_sync(0xffffffffu, v[k], o);
            v[k] = k == 1 ? fmax(v[k], x) : v[k] + x;
        }
    }
    if (l == 0) {
        double *o = part + (size_t)p * NSTAT;
#pragma unroll
        for (int k = 0; k < NSTAT; ++k) o[k] = v[k];
    }
}

// One CTA: fixed strided assignment of pairs to threads, then a fixed tree.
__global__ void __launch_bounds__(1024) k_stats_final(const double *__restrict__ part, uint32_t npairs,
                                                      double *out) {
    __shared__ double red[32];
    double acc[NSTAT] = {0, 0, 0, 0, 0, 0};
    for (uint32_t p = threadIdx.x; p < npairs; p += blockDim.x) {
        const double *o = part + (size_t)p * NSTAT;
        acc[0] += o[0];
        acc[1] = fmax(acc[1], o[1]);
        acc[2] += o[2];
        acc[3] += o[3];
        acc[4] += o[4];
        acc[5] += o[5];
    }
    double r[NSTAT];
    r[0] = block_sum(acc[0], red);
    r[1] = block_max(acc[1], red);
    r[2] = block_sum(acc[2], red);
    r[3] = block_sum(acc[3], red);
    r[4] = block_sum(acc[4], red);
    r[5] = block_sum(acc[5], red);
    if (threadIdx.x == 0) {
        out[0] = r[0];
        out[1] = r[1];
        out[2] = r[3] > 0 ? r[2] / r[3] : 0.0;
        out[3] = r[3];
        out[4] = r[4];
        out[5] = r[5];
    }
}

}  // namespace mi3

using namespace mi3;

extern "C" size_t mi3_gauge_workspace(uint32_t L, uint32_t q) {
    const uint64_t np = npairs_of(L);
    return (size_t)(np * (2ull * q + 1) + (uint64_t)L * q) * sizeof(double);
}

extern "C" int mi3_gauge_fieldless_even(const float *J, float *Jout, uint32_t L, uint32_t q, void *workspace,
                                        size_t ws_bytes, void *stream) {
    if (!J || !Jout || !workspace) return fail(MI3_ERR_ARG, "mi3_gauge_fieldless_even: null pointer");
    if (L < 2 || q < 1 || q > 255) return fail(MI3_ERR_ARG, "mi3_gauge_fieldless_even: bad L/q");
    if (ws_bytes < mi3_gauge_workspace(L, q))
        return fail(MI3_ERR_WORKSPACE, "mi3_gauge_fieldless_even: workspace too small");
    if (!aligned(workspace, 8)) return fail(MI3_ERR_ALIGN, "mi3_gauge_fieldless_even: workspace alignment");
    const uint64_t np = npairs_of(L);
    if (np > 0x7fffffffull) return fail(MI3_ERR_ARG, "mi3_gauge_fieldless_even: L too large");
    cudaStream_t st = as_stream(stream);
    double *m1 = reinterpret_cast<double *>(workspace);
    double *m2 = m1 + np * q;
    double *mJ = m2 + np * q;
    double *hd = mJ + np;
    if (q <= 32) {
        k_gauge_means_w<<<(uint32_t)((np + 7) / 8), 256, 0, st>>>(J, m1, m2, mJ, q, (uint32_t)np);
    } else {
        const uint32_t thr = q <= 128 ? 128 : 256;
        k_gauge_means<<<(uint32_t)np, thr, 0, st>>>(J, m1, m2, mJ, q);
    }
    int rc = check_launch("mi3_gauge_fieldless_even: means");
    if (rc) return rc;
    if (q <= 32)
        k_gauge_fields_w<<<L, 256, 0, st>>>(m1, m2, mJ, hd, L, q);
    else
        k_gauge_fields<<<L, q <= 128 ? 128 : 256, 0, st>>>(m1, m2, mJ, hd, L, q);
    rc = check_launch("mi3_gauge_fieldless_even: fields");
    if (rc) return rc;
    if (q <= 32)
        k_gauge_apply_w<<<(uint32_t)((np + 7) / 8), 256, 0, st>>>(J, Jout, m1, m2, mJ, hd, L, q, (uint32_t)np);
    else
        k_gauge_apply<<<(uint32_t)np, 256, 0, st>>>(J, Jout, m1, m2, mJ, hd, L, q);
    return check_launch("mi3_gauge_fieldless_even: apply");
}

extern "C" size_t mi3_bimarg_stats_workspace(uint32_t L) { return (size_t)npairs_of(L) * NSTAT * sizeof(double); }

extern "C" int mi3_bimarg_stats(const float *target, const float *model, const float *J, uint32_t L, uint32_t q,
                                double *out, void *workspace, size_t ws_bytes, void *stream) {
    if (!target || !model || !out || !workspace) return fail(MI3_ERR_ARG, "mi3_bimarg_stats: null pointer");
    if (L < 2 || q < 1 || q > 255) return fail(MI3_ERR_ARG, "mi3_bimarg_stats: bad L/q");
    if (ws_bytes < mi3_bimarg_stats_workspace(L))
        return fail(MI3_ERR_WORKSPACE, "mi3_bimarg_stats: workspace too small");
    if (!aligned(workspace, 8) || !aligned(out, 8)) return fail(MI3_ERR_ALIGN, "mi3_bimarg_stats: alignment");
    const uint64_t np = npairs_of(L);
    if (np > 0x7fffffffull) return fail(MI3_ERR_ARG, "mi3_bimarg_stats: L too large");
    cudaStream_t st = as_stream(stream);
    double *part = reinterpret_cast<double *>(workspace);
    if (q <= 32) {
        const size_t sm = (size_t)8 * 2 * q * q * sizeof(float);
        if (sm > 40 * 1024) cudaFuncSetAttribute(k_pair_stats_w, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k_pair_stats_w<<<(uint32_t)((np + 7) / 8), 256, sm, st>>>(target, model, J, part, q, (uint32_t)np);
    }
    else
        k_pair_stats<<<(uint32_t)np, STAT_THREADS, 4 * q * sizeof(double), st>>>(target, model, J, part, q);
    int rc = check_launch("mi3_bimarg_stats: pairs");
    if (rc) return rc;
    k_stats_final<<<1, 1024, 0, st>>>(part, (uint32_t)np, out);
    return check_launch("mi3_bimarg_stats: final");
}
