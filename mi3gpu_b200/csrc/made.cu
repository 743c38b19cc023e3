// made.cu -- learned autoregressive proposal: a MADE network (masked MLP
// over L sites x q residues, two hidden layers of H units) with hand-written
// forward, backward, Adam and sampling kernels, and the independence
// Metropolis-Hastings step that uses it.
//
// Parameters (row-major, float32 master copies; the network computes with
// weights rounded to bf16, stored as bf16 for the sampler and as their exact
// float values for training, accumulating in float32):
//   W1T [Lq][H]  input (site i, residue a) -> hidden-1 unit k   (transposed)
//   b1  [H]
//   W2  [H][H]   hidden-1 unit k -> hidden-2 unit k'  (W2[k'][k])
//   b2  [H]
//   W3  [Lq][H]  hidden-2 unit k' -> output (site i, residue a)
//   b3  [Lq]
// MADE masks (degrees m1, m2 in [1, L-1], input/output degree of site i is
// i+1) are applied by keeping masked weights and their gradients at zero, so
// output site i depends on sites < i only.
#include <cuda_bf16.h>

#include <algorithm>

#include "made.cuh"

namespace mi3 {

// --------------------------------------------------------------- SIMT GEMM
// C[m][n] = alpha * sum_k A(m,k) B(k,n) + beta * C[m][n]
// A(m,k) = A[m*sam + k*sak], B(k,n) = B[k*sbk + n*sbn]; C row-major ldc.
constexpr int GT = 64, GK = 16;

__global__ void __launch_bounds__(256) k_gemm(int M, int N, int K, const float *__restrict__ A, long sam, long sak,
                                              const float *__restrict__ B, long sbk, long sbn, float *C, long ldc,
                                              float alpha, float beta) {
    __shared__ float As[GK][GT + 4];
    __shared__ float Bs[GK][GT + 4];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const int m0 = blockIdx.y * GT, n0 = blockIdx.x * GT;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += GK) {
        for (int e = threadIdx.x; e < GT * GK; e += 256) {
            int mm = e / GK, kk = e % GK;  // A tile: 64 rows x 16 k
            int gm = m0 + mm, gk = k0 + kk;
            As[kk][mm] = (gm < M && gk < K) ? A[gm * sam + gk * sak] : 0.0f;
            int kb = e / GT, nn = e % GT;  // B tile: 16 k x 64 cols
            int gk2 = k0 + kb, gn = n0 + nn;
            Bs[kb][nn] = (gk2 < K && gn < N) ? B[gk2 * sbk + gn * sbn] : 0.0f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < GK; ++kk) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        int gm = m0 + ty * 4 + i;
        if (gm >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            int gn = n0 + tx * 4 + j;
            if (gn >= N) continue;
            float *c = &C[gm * ldc + gn];
            *c = alpha * acc[i][j] + (beta != 0.0f ? beta * *c : 0.0f);
        }
    }
}

// Where the dense products run: the FP32 SIMT kernel above (ws null), or
// the BF16 tensor-core GEMM (mi3_gemm_bf16) with its workspace.
struct GemmPath {
    void *ws = nullptr;
    uint64_t ws_bytes = 0;
    int32_t *status = nullptr;
};

static int gemm(const GemmPath &gp, int M, int N, int K, const float *A, long sam, long sak, const float *B, long sbk,
                long sbn, float *C, long ldc, float alpha, float beta, cudaStream_t st) {
    if (gp.ws)
        return mi3_gemm_bf16(M, N, K, A, sam, sak, B, sbk, sbn, C, ldc, alpha, beta, gp.ws, gp.ws_bytes, gp.status,
                             st);
    dim3 grid((N + GT - 1) / GT, (M + GT - 1) / GT);
    k_gemm<<<grid, 256, 0, st>>>(M, N, K, A, sam, sak, B, sbk, sbn, C, ldc, alpha, beta);
    return check_launch("made gemm");
}

__device__ __forceinline__ uint32_t seq_res(const uint32_t *seq, uint32_t buflen, uint32_t n, uint32_t i) {
    return (seq[(size_t)(i >> 2) * buflen + n] >> (8 * (i & 3))) & 0xffu;
}

// h1[b][k] = b1[k] + sum_i W1T[i*q + s_i][k]
__global__ void k_made_h1(const uint32_t *__restrict__ seq, uint32_t buflen, uint32_t n0, int B, int L, int q, int H,
                          const float *__restrict__ W1T, const float *__restrict__ b1, float *h1) {
    int b = blockIdx.y;
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B || k >= H) return;
    float acc = b1[k];
    for (int i = 0; i < L; ++i) {
        uint32_t a = min(seq_res(seq, buflen, n0 + b, i), (uint32_t)(q - 1));
        acc += W1T[(size_t)(i * q + a) * H + k];
    }
    h1[(size_t)b * H + k] = acc;
}

__global__ void k_relu(const float *__restrict__ x, float *y, size_t n) {
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) y[t] = fmaxf(x[t], 0.0f);
}

__global__ void k_add_bias(float *x, const float *__restrict__ bias, int rows, int cols) {
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < (size_t)rows * cols) x[t] += bias[t % cols];
}

// Per sequence: log q = sum over sites of the log softmax of the q logits at
// the observed residue; optionally dlogits = (softmax - onehot) * scale.
__global__ void k_made_loss(const uint32_t *__restrict__ seq, uint32_t buflen, uint32_t n0, int B, int L, int q,
                            const float *__restrict__ logits, float *logq, float *dlogits, float scale) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    const int Lq = L * q;
    double lq = 0.0;
    for (int i = 0; i < L; ++i) {
        const float *o = logits + (size_t)b * Lq + i * q;
        float mx = o[0];
        for (int a = 1; a < q; ++a) mx = fmaxf(mx, o[a]);
        float se = 0.0f;
        for (int a = 0; a < q; ++a) se += expf(o[a] - mx);
        float lse = mx + logf(se);
        uint32_t s = min(seq_res(seq, buflen, n0 + b, i), (uint32_t)(q - 1));
        lq += (double)(o[s] - lse);
        if (dlogits) {
            float *d = dlogits + (size_t)b * Lq + i * q;
            for (int a = 0; a < q; ++a) d[a] = (expf(o[a] - lse) - (a == (int)s ? 1.0f : 0.0f)) * scale;
        }
    }
    if (logq) logq[b] = (float)lq;
}

// g = g * (pre > 0)
__global__ void k_relu_grad(const float *__restrict__ pre, float *g, size_t n) {
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n && !(pre[t] > 0.0f)) g[t] = 0.0f;
}

// column sums: out[c] = sum_r x[r][c] (+ beta * out[c])
__global__ void k_colsum(const float *__restrict__ x, int rows, int cols, float *out, float beta) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float s = 0.0f;
    for (int r = 0; r < rows; ++r) s += x[(size_t)r * cols + c];
    out[c] = s + (beta != 0.0f ? beta * out[c] : 0.0f);
}

// X[b][i*q + a] = [s_i == a]
__global__ void k_onehot(const uint32_t *__restrict__ seq, uint32_t buflen, uint32_t n0, int B, int L, int q,
                         float *X) {
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t Lq = (size_t)L * q;
    if (t >= (size_t)B * Lq) return;
    int b = (int)(t / Lq);
    int c = (int)(t % Lq);
    int i = c / q, a = c % q;
    X[t] = (seq_res(seq, buflen, n0 + b, i) == (uint32_t)a) ? 1.0f : 0.0f;
}

__global__ void k_mask_mul(float *g, const float *__restrict__ mask, size_t n) {
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) g[t] *= mask[t];
}

// Adam on one parameter block; master p (float32), the bf16-rounded compute
// copy pc (float) and the bf16 copy ph are refreshed; masked entries stay 0.
__global__ void k_adam(float *p, float *pc, __nv_bfloat16 *ph, const float *__restrict__ g, float *m, float *v,
                       const float *__restrict__ mask, size_t n, float lr, float b1, float b2, float eps, float c1,
                       float c2) {
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    float gt = g[t];
    float mt = b1 * m[t] + (1.0f - b1) * gt;
    float vt = b2 * v[t] + (1.0f - b2) * gt * gt;
    m[t] = mt;
    v[t] = vt;
    float pt = p[t] - lr * (mt / c1) / (sqrtf(vt / c2) + eps);
    if (mask && mask[t] == 0.0f) pt = 0.0f;
    p[t] = pt;
    __nv_bfloat16 h = __float2bfloat16_rn(pt);
    if (ph) ph[t] = h;
    pc[t] = __bfloat162float(h);
}

__global__ void k_round_bf16(const float *__restrict__ p, float *pc, __nv_bfloat16 *ph, size_t n) {
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    __nv_bfloat16 h = __float2bfloat16_rn(p[t]);
    if (ph) ph[t] = h;
    pc[t] = __bfloat162float(h);
}

// ------------------------------------------------------------- sampling
constexpr int SAMP_S = 32;  // sequences per CTA (one per lane)
constexpr int NWARP = 8;    // warps per CTA (256 threads)

// Autoregressive sampling in MADE degree order.  Hidden-1 unit k with degree
// m1 depends on sites < m1, hidden-2 unit k' with degree m2 on hidden-1 units
// with m1 <= m2, output site i on hidden-2 units with m2 <= i.  Walking the
// sites in order, a hidden-1 pre-activation is a running sum (one column of
// W1T added per drawn site) and each hidden-2 unit is evaluated exactly
// once, at the step where its degree is reached: one forward pass per
// sequence instead of L.  deg2_start[d]..deg2_start[d+1] index the hidden-2
// units of degree d in deg2_units.  With `given` set the residues are read
// from `seq` instead of drawn (teacher forcing: log q of given sequences).
__global__ void __launch_bounds__(256) k_made_sample(int L, int q, int H, const __nv_bfloat16 *__restrict__ W1T,
                                                     const float *__restrict__ b1, const __nv_bfloat16 *__restrict__ W2,
                                                     const float *__restrict__ b2, const __nv_bfloat16 *__restrict__ W3,
                                                     const float *__restrict__ b3, const int *__restrict__ deg2_start,
                                                     const int *__restrict__ deg2_units, uint32_t *seq_out,
                                                     uint32_t buflen, uint32_t nseq, float *logq, uint64_t seed,
                                                     int given) {
    extern __shared__ float sm[];
    // rows padded to H+1 floats: lane s of a warp reads row s, and a stride
    // of H+1 puts the 32 lanes in 32 different banks
    const int HP = H + 1;
    float *h1 = sm;                      // [S][H+1] hidden-1 pre-activations
    float *h2 = h1 + SAMP_S * HP;        // [S][H+1] hidden-2 activations (0 until evaluated)
    float *lg = h2 + SAMP_S * HP;        // [S][33] logits of the current site
    uint32_t *res = reinterpret_cast<uint32_t *>(lg + SAMP_S * 33);  // [S] residue just chosen
    float *lq = reinterpret_cast<float *>(res + SAMP_S);             // [S] log q accumulator
    float *red = lq + SAMP_S;                                        // [8 warps][4][S] partial sums
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int KC = (H + NWARP - 1) / NWARP;
    const uint32_t nbase = blockIdx.x * SAMP_S;

    for (int e = tid; e < SAMP_S * H; e += nthr) {
        const int s = e / H, k = e % H;
        h1[s * HP + k] = b1[k];
        h2[s * HP + k] = 0.0f;
    }
    if (tid < SAMP_S) lq[tid] = 0.0f;
    __syncthreads();

    for (int i = 0; i < L; ++i) {
        // (a) hidden-2 units of degree i (all their hidden-1 inputs are final).
        // Warp w sums inputs k in [w*KC, (w+1)*KC) for sequence s = lane, four
        // units at a time; the 8 partial sums are then added in warp order.
        const int u0 = deg2_start[i], u1 = deg2_start[i + 1];
        for (int ug = u0; ug < u1; ug += 4) {
            const int nu = min(4, u1 - ug);
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
            const float *x = h1 + lane * HP;
            const int kb = warp * KC, ke = min(H, kb + KC);
            int uu[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) uu[j] = deg2_units[ug + min(j, nu - 1)];
            for (int k = kb; k < ke; ++k) {
                const float xv = fmaxf(x[k], 0.0f);
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[j] = fmaf(__bfloat162float(W2[(size_t)uu[j] * H + k]), xv, acc[j]);
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) red[(warp * 4 + j) * SAMP_S + lane] = acc[j];
            __syncthreads();
            if (tid < 4 * SAMP_S) {
                const int j = tid / SAMP_S, sq = tid % SAMP_S;
                if (j < nu) {
                    float v = b2[uu[j]];
                    for (int w = 0; w < NWARP; ++w) v += red[(w * 4 + j) * SAMP_S + sq];
                    h2[sq * HP + uu[j]] = fmaxf(v, 0.0f);
                }
            }
            __syncthreads();
        }
        // (b) logits of site i, four residues at a time, same split
        for (int ag = 0; ag < q; ag += 4) {
            const int na = min(4, q - ag);
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
            const float *x = h2 + lane * HP;
            const int kb = warp * KC, ke = min(H, kb + KC);
            for (int k = kb; k < ke; ++k) {
                const float xv = x[k];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int a = ag + min(j, na - 1);
                    acc[j] = fmaf(__bfloat162float(W3[(size_t)(i * q + a) * H + k]), xv, acc[j]);
                }
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) red[(warp * 4 + j) * SAMP_S + lane] = acc[j];
            __syncthreads();
            if (tid < 4 * SAMP_S) {
                const int j = tid / SAMP_S, sq = tid % SAMP_S;
                if (j < na) {
                    float v = b3[i * q + ag + j];
                    for (int w = 0; w < NWARP; ++w) v += red[(w * 4 + j) * SAMP_S + sq];
                    lg[sq * 33 + ag + j] = v;
                }
            }
            __syncthreads();
        }
        // (c) draw (or read) residue i, accumulate log q
        if (tid < SAMP_S) {
            const int s = tid;
            const uint32_t n = nbase + s;
            const float *o = lg + s * 33;
            float mx = o[0];
            for (int a = 1; a < q; ++a) mx = fmaxf(mx, o[a]);
            float se = 0.0f;
            for (int a = 0; a < q; ++a) se += expf(o[a] - mx);
            const float lse = mx + logf(se);
            uint32_t r;
            if (given) {
                r = (n < nseq) ? min(seq_res(seq_out, buflen, n, i), (uint32_t)(q - 1)) : 0u;
            } else {
                const float u = hash_uniform(seed, n, i) * se;
                float c = 0.0f;
                r = q - 1;
                for (int a = 0; a < q; ++a) {
                    c += expf(o[a] - mx);
                    if (u < c) {
                        r = a;
                        break;
                    }
                }
            }
            res[s] = r;
            lq[s] += o[r] - lse;
            if (!given && n < nseq) {
                uint32_t *wp = seq_out + (size_t)(i >> 2) * buflen + n;
                uint32_t sh = 8 * (i & 3);
                uint32_t wv = (i & 3) ? *wp : 0u;  // the first site of a word clears it
                *wp = (wv & ~(0xffu << sh)) | (r << sh);
            }
        }
        __syncthreads();
        // (d) add the chosen residue's column to every hidden-1 unit
        for (int e = tid; e < SAMP_S * H; e += nthr) {
            const int s = e / H, k = e % H;
            h1[s * HP + k] += __bfloat162float(W1T[(size_t)(i * q + res[s]) * H + k]);
        }
        __syncthreads();
    }
    if (tid < SAMP_S && nbase + tid < nseq) logq[nbase + tid] = lq[tid];
}

// Independence Metropolis-Hastings: accept the proposal with probability
// min(1, exp(-(E' - E)) q(s) / q(s')).  Accepted walkers copy the proposal's
// words and values; counts acceptances.
__global__ void k_mh_accept(uint32_t *seq, const uint32_t *__restrict__ prop, uint32_t buflen, uint32_t nseq,
                            uint32_t swords, float *E, const float *__restrict__ Ep, float *lq,
                            const float *__restrict__ lqp, uint64_t seed, unsigned long long *naccept) {
    uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    bool acc = false;
    if (n < nseq) {
        float logr = -(Ep[n] - E[n]) + (lq[n] - lqp[n]);
        float u = hash_uniform(seed, n, 0xFFFFFFFFull);
        acc = (logr >= 0.0f) || (u < expf(logr));
        if (acc) {
            for (uint32_t w = 0; w < swords; ++w) seq[(size_t)w * buflen + n] = prop[(size_t)w * buflen + n];
            E[n] = Ep[n];
            lq[n] = lqp[n];
        }
    }
    unsigned int ball = __ballot_sync(0xffffffffu, acc);
    if ((threadIdx.x & 31) == 0 && ball) atomicAdd(naccept, (unsigned long long)__popc(ball));
}

static inline unsigned nb(size_t n, unsigned t = 256) { return (unsigned)((n + t - 1) / t); }

}  // namespace mi3

using namespace mi3;

// --------------------------------------------------------------- C ABI
static int made_forward(const GemmPath &gp, const uint32_t *seq, uint32_t buflen, uint32_t n0, uint32_t B, uint32_t L,
                                uint32_t q, uint32_t H, const float *W1T, const float *b1, const float *W2,
                                const float *b2, const float *W3, const float *b3, float *h1, float *a1, float *h2,
                                float *a2, float *logits, float *logq, void *stream) {
    if (!seq || !W1T || !b1 || !W2 || !b2 || !W3 || !b3 || !h1 || !a1 || !h2 || !a2 || !logits)
        return fail(MI3_ERR_ARG, "mi3_made_forward: null pointer");
    if (B == 0 || L < 2 || q < 2 || q > 32 || H == 0 || n0 + B > buflen)
        return fail(MI3_ERR_ARG, "mi3_made_forward: bad sizes");
    cudaStream_t st = as_stream(stream);
    const int Lq = L * q;
    dim3 g1(nb(H), B);
    k_made_h1<<<g1, 256, 0, st>>>(seq, buflen, n0, B, L, q, H, W1T, b1, h1);
    k_relu<<<nb((size_t)B * H), 256, 0, st>>>(h1, a1, (size_t)B * H);
    // h2 = a1 W2^T + b2
    int rc = gemm(gp, B, H, H, a1, H, 1, W2, 1, H, h2, H, 1.0f, 0.0f, st);
    if (rc) return rc;
    k_add_bias<<<nb((size_t)B * H), 256, 0, st>>>(h2, b2, B, H);
    k_relu<<<nb((size_t)B * H), 256, 0, st>>>(h2, a2, (size_t)B * H);
    rc = gemm(gp, B, Lq, H, a2, H, 1, W3, 1, H, logits, Lq, 1.0f, 0.0f, st);
    if (rc) return rc;
    k_add_bias<<<nb((size_t)B * Lq), 256, 0, st>>>(logits, b3, B, Lq);
    if (logq) k_made_loss<<<nb(B, 128), 128, 0, st>>>(seq, buflen, n0, B, L, q, logits, logq, nullptr, 0.0f);
    return check_launch("mi3_made_forward");
}

static int made_backward(const GemmPath &gp, const uint32_t *seq, uint32_t buflen, uint32_t n0, uint32_t B, uint32_t L,
                                 uint32_t q, uint32_t H, const float *W2, const float *W3, const float *h1,
                                 const float *a1, const float *h2, const float *a2, const float *logits,
                                 float *dlogits, float *X, float *dh1, float *dh2, float *gW1T, float *gb1, float *gW2,
                                 float *gb2, float *gW3, float *gb3, const float *mW1T, const float *mW2,
                                 const float *mW3, float *loss_per_seq, void *stream) {
    if (!seq || !W2 || !W3 || !h1 || !a1 || !h2 || !a2 || !logits || !dlogits || !X || !dh1 || !dh2 || !gW1T ||
        !gb1 || !gW2 || !gb2 || !gW3 || !gb3 || !mW1T || !mW2 || !mW3)
        return fail(MI3_ERR_ARG, "mi3_made_backward: null pointer");
    if (B == 0 || L < 2 || q < 2 || q > 32 || H == 0 || n0 + B > buflen)
        return fail(MI3_ERR_ARG, "mi3_made_backward: bad sizes");
    cudaStream_t st = as_stream(stream);
    const int Lq = L * q;
    k_made_loss<<<nb(B, 128), 128, 0, st>>>(seq, buflen, n0, B, L, q, logits, loss_per_seq, dlogits, 1.0f / B);
    int rc;
    // gW3[o][k'] = sum_b dlogits[b][o] a2[b][k']
    if ((rc = gemm(gp, Lq, H, B, dlogits, 1, Lq, a2, H, 1, gW3, H, 1.0f, 0.0f, st))) return rc;
    k_colsum<<<nb(Lq), 256, 0, st>>>(dlogits, B, Lq, gb3, 0.0f);
    // dh2 = dlogits W3 * relu'(h2)
    if ((rc = gemm(gp, B, H, Lq, dlogits, Lq, 1, W3, H, 1, dh2, H, 1.0f, 0.0f, st))) return rc;
    k_relu_grad<<<nb((size_t)B * H), 256, 0, st>>>(h2, dh2, (size_t)B * H);
    // gW2[k'][k] = sum_b dh2[b][k'] a1[b][k]
    if ((rc = gemm(gp, H, H, B, dh2, 1, H, a1, H, 1, gW2, H, 1.0f, 0.0f, st))) return rc;
    k_colsum<<<nb(H), 256, 0, st>>>(dh2, B, H, gb2, 0.0f);
    // dh1 = dh2 W2 * relu'(h1)
    if ((rc = gemm(gp, B, H, H, dh2, H, 1, W2, H, 1, dh1, H, 1.0f, 0.0f, st))) return rc;
    k_relu_grad<<<nb((size_t)B * H), 256, 0, st>>>(h1, dh1, (size_t)B * H);
    // gW1T[(i,a)][k] = sum_b X[b][(i,a)] dh1[b][k]
    k_onehot<<<nb((size_t)B * Lq), 256, 0, st>>>(seq, buflen, n0, B, L, q, X);
    if ((rc = gemm(gp, Lq, H, B, X, 1, Lq, dh1, H, 1, gW1T, H, 1.0f, 0.0f, st))) return rc;
    k_colsum<<<nb(H), 256, 0, st>>>(dh1, B, H, gb1, 0.0f);
    k_mask_mul<<<nb((size_t)Lq * H), 256, 0, st>>>(gW1T, mW1T, (size_t)Lq * H);
    k_mask_mul<<<nb((size_t)H * H), 256, 0, st>>>(gW2, mW2, (size_t)H * H);
    k_mask_mul<<<nb((size_t)Lq * H), 256, 0, st>>>(gW3, mW3, (size_t)Lq * H);
    return check_launch("mi3_made_backward");
}

extern "C" int mi3_made_forward(const uint32_t *seq, uint32_t buflen, uint32_t n0, uint32_t B, uint32_t L,
                                uint32_t q, uint32_t H, const float *W1T, const float *b1, const float *W2,
                                const float *b2, const float *W3, const float *b3, float *h1, float *a1, float *h2,
                                float *a2, float *logits, float *logq, void *stream) {
    return made_forward(GemmPath{}, seq, buflen, n0, B, L, q, H, W1T, b1, W2, b2, W3, b3, h1, a1, h2, a2, logits, logq,
                        stream);
}

extern "C" int mi3_made_backward(const uint32_t *seq, uint32_t buflen, uint32_t n0, uint32_t B, uint32_t L,
                                 uint32_t q, uint32_t H, const float *W2, const float *W3, const float *h1,
                                 const float *a1, const float *h2, const float *a2, const float *logits,
                                 float *dlogits, float *X, float *dh1, float *dh2, float *gW1T, float *gb1, float *gW2,
                                 float *gb2, float *gW3, float *gb3, const float *mW1T, const float *mW2,
                                 const float *mW3, float *loss_per_seq, void *stream) {
    return made_backward(GemmPath{}, seq, buflen, n0, B, L, q, H, W2, W3, h1, a1, h2, a2, logits, dlogits, X, dh1,
                         dh2, gW1T, gb1, gW2, gb2, gW3, gb3, mW1T, mW2, mW3, loss_per_seq, stream);
}

extern "C" uint64_t mi3_made_gemm_workspace(uint32_t B, uint32_t L, uint32_t q, uint32_t H) {
    const uint32_t Lq = L * q;
    uint64_t w = 0;
    const uint32_t shapes[7][3] = {{B, H, H}, {B, Lq, H}, {Lq, H, B}, {B, H, Lq}, {H, H, B}, {B, H, H}, {Lq, H, B}};
    for (const auto &sh : shapes) w = std::max<uint64_t>(w, mi3_gemm_bf16_workspace(sh[0], sh[1], sh[2]));
    return w;
}

extern "C" int mi3_made_forward_tc(const uint32_t *seq, uint32_t buflen, uint32_t n0, uint32_t B, uint32_t L,
                                   uint32_t q, uint32_t H, const float *W1T, const float *b1, const float *W2,
                                   const float *b2, const float *W3, const float *b3, float *h1, float *a1, float *h2,
                                   float *a2, float *logits, float *logq, void *workspace, uint64_t ws_bytes,
                                   int32_t *status, void *stream) {
    if (!workspace || !status) return fail(MI3_ERR_ARG, "mi3_made_forward_tc: null workspace or status");
    GemmPath gp{workspace, ws_bytes, status};
    return made_forward(gp, seq, buflen, n0, B, L, q, H, W1T, b1, W2, b2, W3, b3, h1, a1, h2, a2, logits, logq,
                        stream);
}

extern "C" int mi3_made_backward_tc(const uint32_t *seq, uint32_t buflen, uint32_t n0, uint32_t B, uint32_t L,
                                    uint32_t q, uint32_t H, const float *W2, const float *W3, const float *h1,
                                    const float *a1, const float *h2, const float *a2, const float *logits,
                                    float *dlogits, float *X, float *dh1, float *dh2, float *gW1T, float *gb1,
                                    float *gW2, float *gb2, float *gW3, float *gb3, const float *mW1T,
                                    const float *mW2, const float *mW3, float *loss_per_seq, void *workspace,
                                    uint64_t ws_bytes, int32_t *status, void *stream) {
    if (!workspace || !status) return fail(MI3_ERR_ARG, "mi3_made_backward_tc: null workspace or status");
    GemmPath gp{workspace, ws_bytes, status};
    return made_backward(gp, seq, buflen, n0, B, L, q, H, W2, W3, h1, a1, h2, a2, logits, dlogits, X, dh1, dh2, gW1T,
                         gb1, gW2, gb2, gW3, gb3, mW1T, mW2, mW3, loss_per_seq, stream);
}

extern "C" int mi3_made_adam(float *p, float *pc, void *ph_bf16, const float *g, float *m, float *v, const float *mask,
                             uint64_t n, float lr, float beta1, float beta2, float eps, uint32_t step, void *stream) {
    if (!p || !pc || !g || !m || !v) return fail(MI3_ERR_ARG, "mi3_made_adam: null pointer");
    if (step == 0) return fail(MI3_ERR_ARG, "mi3_made_adam: step counts from 1");
    float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
    k_adam<<<nb(n), 256, 0, as_stream(stream)>>>(p, pc, reinterpret_cast<__nv_bfloat16 *>(ph_bf16), g, m, v, mask, n,
                                                   lr, beta1, beta2, eps, c1, c2);
    return check_launch("mi3_made_adam");
}

extern "C" int mi3_made_round_bf16(const float *p, float *pc, void *ph_bf16, uint64_t n, void *stream) {
    if (!p || !pc) return fail(MI3_ERR_ARG, "mi3_made_round_bf16: null pointer");
    k_round_bf16<<<nb(n), 256, 0, as_stream(stream)>>>(p, pc, reinterpret_cast<__nv_bfloat16 *>(ph_bf16), n);
    return check_launch("mi3_made_round_bf16");
}

extern "C" int mi3_made_sample(uint32_t L, uint32_t q, uint32_t H, const void *W1T_bf16, const float *b1,
                               const void *W2_bf16, const float *b2, const void *W3_bf16, const float *b3,
                               const int32_t *deg2_start, const int32_t *deg2_units, uint32_t *seq, uint32_t buflen,
                               uint32_t nseq, float *logq, uint64_t seed, int32_t given, void *stream) {
    if (!W1T_bf16 || !b1 || !W2_bf16 || !b2 || !W3_bf16 || !b3 || !deg2_start || !deg2_units || !seq || !logq)
        return fail(MI3_ERR_ARG, "mi3_made_sample: null pointer");
    if (L < 2 || q < 2 || q > 32 || H == 0 || H > 1024 || nseq > buflen)
        return fail(MI3_ERR_ARG, "mi3_made_sample: bad sizes (q <= 32, H <= 1024)");
    if (nseq == 0) return MI3_OK;
    size_t smem = (size_t)(2 * SAMP_S * (H + 1) + SAMP_S * 33 + 2 * SAMP_S + NWARP * 4 * SAMP_S) * 4;
    if (smem > 227 * 1024) return fail(MI3_ERR_ARG, "mi3_made_sample: H too large");
    cudaFuncSetAttribute(k_made_sample, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_made_sample<<<(nseq + SAMP_S - 1) / SAMP_S, 256, smem, as_stream(stream)>>>(
        L, q, H, reinterpret_cast<const __nv_bfloat16 *>(W1T_bf16), b1,
        reinterpret_cast<const __nv_bfloat16 *>(W2_bf16), b2, reinterpret_cast<const __nv_bfloat16 *>(W3_bf16), b3,
        deg2_start, deg2_units, seq, buflen, nseq, logq, seed, given);
    return check_launch("mi3_made_sample");
}

extern "C" int mi3_mh_independence(uint32_t *seq, const uint32_t *prop, uint32_t buflen, uint32_t nseq, uint32_t L,
                                   float *E, const float *Ep, float *logq, const float *logq_prop, uint64_t seed,
                                   unsigned long long *naccept, void *stream) {
    if (!seq || !prop || !E || !Ep || !logq || !logq_prop || !naccept)
        return fail(MI3_ERR_ARG, "mi3_mh_independence: null pointer");
    if (nseq > buflen || L < 1) return fail(MI3_ERR_ARG, "mi3_mh_independence: bad sizes");
    if (nseq == 0) return MI3_OK;
    k_mh_accept<<<nb(nseq), 256, 0, as_stream(stream)>>>(seq, prop, buflen, nseq, (L - 1) / 4 + 1, E, Ep, logq,
                                                          logq_prop, seed, naccept);
    return check_launch("mi3_mh_independence");
}
