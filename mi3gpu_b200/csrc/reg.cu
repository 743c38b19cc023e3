// reg.cu -- the remaining coupling regularizers of the quasi-Newton step
// (mcmc.cl:904-1243): SCADJ, X, Xij, SCADX, expX, ddE, SCADddE.
//
// One warp per pair block (q*q couplings).  Every block-wide sum follows the
// reference's odd-aware reduction tree (sumqq, getUnimarg, zeroGauge), and
// every expression keeps the reference's operation order, so results agree
// bit for bit with a strict float evaluation of mcmc.cl (expX up to expf).
#include "common.cuh"

namespace mi3 {

enum RegKind : int { R_SCADJ = 0, R_X = 1, R_XIJ = 2, R_SCADX = 3, R_EXPX = 4, R_DDE = 5, R_SCADDDE = 6 };

__device__ __forceinline__ float ocl_sign_r(float x) {
    if (x > 0.0f) return 1.0f;
    if (x < 0.0f) return -1.0f;
    if (x != x) return 0.0f;
    return x;
}

__device__ __forceinline__ void rows_tree_w(float *sc, uint32_t q, uint32_t lane) {
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

// sum of sc[0..qq) by the sumqq tree (mcmc.cl:732-751); sc is clobbered.
__device__ __forceinline__ float sumqq_w(float *sc, uint32_t qq, uint32_t lane) {
    __syncwarp();
    uint32_t m = qq;
    while (m > 1) {
        uint32_t odd = m & 1;
        m = (m + 1) >> 1;
        for (uint32_t li = lane; li < m - odd; li += 32) sc[li] = sc[li] + sc[li + m];
        __syncwarp();
    }
    float r = sc[0];
    __syncwarp();
    return r;
}

template <int KIND>
__global__ void k_reg_other(const float *__restrict__ bi, const float *__restrict__ lambdas, float gamma, float pc,
                            float p0, float p1, float p2, const float *__restrict__ J, float *dJ, uint64_t npairs,
                            uint32_t q) {
    extern __shared__ float sm[];
    const uint32_t qq = q * q;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t wpb = blockDim.x >> 5;
    float *sc = sm + warp * (4 * qq + 2 * q + 4);
    float *Jt = sc + qq;
    float *fij = Jt + qq;
    float *C = fij + qq;
    float *fi = C + qq;  // also hi (SCADJ)
    float *fj = fi + q;  // also hj (SCADJ)
    const float fq = (float)q;
    for (uint64_t p = (uint64_t)blockIdx.x * wpb + warp; p < npairs; p += (uint64_t)gridDim.x * wpb) {
        const uint64_t base = p * qq;
        for (uint32_t li = lane; li < qq; li += 32) {
            Jt[li] = J[base + li] + dJ[base + li];
            fij[li] = bi[base + li];
        }
        __syncwarp();
        float X = 0.0f, Xnorm = 0.0f, mean = 0.0f;
        if (KIND == R_SCADJ) {
            // zeroGauge (mcmc.cl:764-822) on Jt
            for (uint32_t li = lane; li < qq; li += 32) sc[li] = Jt[li];
            __syncwarp();
            rows_tree_w(sc, q, lane);
            for (uint32_t a = lane; a < q; a += 32) fi[a] = sc[q * a] / fq;
            __syncwarp();
            for (uint32_t li = lane; li < qq; li += 32) sc[q * (li % q) + li / q] = Jt[li];
            __syncwarp();
            rows_tree_w(sc, q, lane);
            for (uint32_t b = lane; b < q; b += 32) fj[b] = sc[q * b] / fq;
            __syncwarp();
            uint32_t m = q;
            while (m > 1) {
                uint32_t odd = m & 1;
                m = (m + 1) >> 1;
                for (uint32_t li = lane; li < m - odd; li += 32) sc[q * li] = sc[q * li] + sc[q * (li + m)];
                __syncwarp();
            }
            mean = sc[0] / fq / fq;
            __syncwarp();
            for (uint32_t a = lane; a < q; a += 32) {
                fi[a] = fi[a] - mean;
                fj[a] = fj[a] - mean;
            }
            __syncwarp();
        } else if (KIND <= R_EXPX) {
            // getUnimarg (mcmc.cl:936-973)
            for (uint32_t li = lane; li < qq; li += 32) sc[li] = fij[li];
            __syncwarp();
            rows_tree_w(sc, q, lane);
            for (uint32_t a = lane; a < q; a += 32) fi[a] = sc[q * a];
            __syncwarp();
            for (uint32_t li = lane; li < qq; li += 32) sc[q * (li % q) + li / q] = fij[li];
            __syncwarp();
            rows_tree_w(sc, q, lane);
            for (uint32_t b = lane; b < q; b += 32) fj[b] = sc[q * b];
            __syncwarp();
            for (uint32_t li = lane; li < qq; li += 32) C[li] = fij[li] - fi[li / q] * fj[li % q];
            __syncwarp();
            for (uint32_t li = lane; li < qq; li += 32) sc[li] = Jt[li] * C[li];
            X = sumqq_w(sc, qq, lane);
            if (KIND != R_EXPX) {
                for (uint32_t li = lane; li < qq; li += 32) sc[li] = C[li] * C[li] / (fij[li] + pc);
                Xnorm = sumqq_w(sc, qq, lane);
            }
        }
        for (uint32_t li = lane; li < qq; li += 32) {
            const float Jp = dJ[base + li];
            const float f = fij[li];
            float outv;
            if (KIND == R_SCADJ) {
                float lJ = p0, a = p1;
                float j0 = Jt[li] - (fi[li / q] + fj[li % q]) - mean;
                float R = 0.0f;
                if (fabsf(j0) < lJ) R = fminf(lJ, fabsf(j0) / gamma);
                else if (fabsf(j0) < a * lJ) R = (a * lJ - fabsf(j0)) / (a - 1.0f);
                R *= gamma * ocl_sign_r(j0) / (f + pc);
                outv = Jp - R;
            } else if (KIND == R_X) {
                float lX = fminf(p0, fabsf(X) / (Xnorm * gamma));
                outv = Jp - gamma * lX * C[li] * ocl_sign_r(X) / (f + pc);
            } else if (KIND == R_XIJ) {
                float lX = fminf(lambdas[p], fabsf(X) / (Xnorm * gamma));
                float R = lX * C[li] * ocl_sign_r(X);
                outv = Jp - gamma * R / (f + pc);
            } else if (KIND == R_SCADX || KIND == R_EXPX) {
                const uint32_t c = li / q, d = li % q;
                float xab = 0.0f;
                for (uint32_t a = 0; a < q; a++)
                    for (uint32_t b = 0; b < q; b++)
                        xab += Jt[a * q + b] * (fi[a] - (float)(a == c)) * (fj[b] - (float)(b == d));
                if (KIND == R_SCADX) {
                    float s = p0, r = p1, a = p2;
                    float R = 0.0f;
                    if (fabsf(X) < r) {
                        r = fminf(r, fabsf(X) / (Xnorm * gamma * s));
                        R = r * ocl_sign_r(X);
                    } else if (fabsf(X) < a * r) {
                        R = (a * r * ocl_sign_r(X) - X) / (a - 1.0f);
                    }
                    R *= gamma * s * (C[li] + f * (X - xab)) / (f + pc);
                    outv = Jp - R;
                } else {
                    float R = ocl_sign_r(X) * expf(-fabsf(X) / p0) * (C[li] + f * (X - xab));
                    outv = Jp - gamma * R / (f + pc);
                }
            } else {
                const float lambda = p0, r = p1;
                const uint32_t a = li / q, b = li % q;
                float dR = 0.0f;
                for (uint32_t g = 1; g < q; g++) {
                    float jr = Jt[q * a + b] - Jt[q * ((a + g) % q) + b];
                    for (uint32_t d = 1; d < q; d++) {
                        float jc = -Jt[q * a + (b + d) % q] + Jt[q * ((a + g) % q) + (b + d) % q];
                        float dde = jr + jc;
                        if (KIND == R_DDE) {
                            dR += ocl_sign_r(dde);
                        } else {
                            float R = 0.0f, absD = fabsf(dde);
                            if (absD < r) R = 1.0f;
                            else if (absD < 4.0f * r) R = (4.0f * r - absD) / (4.0f * r - r);
                            dR += lambda * ocl_sign_r(dde) * R;
                        }
                    }
                }
                dR = dR / (float)((q - 1) * (q - 1));
                if (KIND == R_DDE) outv = Jp - lambda * dR * gamma / (f + pc);
                else outv = Jp - gamma * dR / (f + pc);
            }
            dJ[base + li] = outv;
        }
        __syncwarp();
    }
}

template <int KIND>
static int launch_reg(const char *name, const float *bi, const float *lambdas, float gamma, float pc, float p0,
                      float p1, float p2, const float *J, float *dJ, uint32_t L, uint32_t q, void *stream) {
    if (!bi || !J || !dJ || (KIND == R_XIJ && !lambdas)) return fail(MI3_ERR_ARG, std::string(name) + ": null pointer");
    if (L < 2 || q < 2 || q > 32) return fail(MI3_ERR_ARG, std::string(name) + ": bad L/q (2 <= q <= 32)");
    uint64_t np = npairs_of(L);
    const uint32_t tb = 256;
    size_t smem = (size_t)(tb / 32) * (4 * q * q + 2 * q + 4) * 4;
    cudaFuncSetAttribute(k_reg_other<KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    uint32_t grid = (uint32_t)std::min<uint64_t>((np + 7) / 8, 148 * 16);
    k_reg_other<KIND><<<grid, tb, smem, as_stream(stream)>>>(bi, lambdas, gamma, pc, p0, p1, p2, J, dJ, np, q);
    return check_launch(name);
}

}  // namespace mi3

using namespace mi3;

extern "C" int mi3_reg_scadj(const float *bi, float gamma, float pc, float lJ, float a, const float *J, float *dJ,
                             uint32_t L, uint32_t q, void *stream) {
    return launch_reg<R_SCADJ>("mi3_reg_scadj", bi, nullptr, gamma, pc, lJ, a, 0.f, J, dJ, L, q, stream);
}

extern "C" int mi3_reg_x(const float *bi, float lX, float gamma, float pc, const float *J, float *dJ, uint32_t L,
                         uint32_t q, void *stream) {
    return launch_reg<R_X>("mi3_reg_x", bi, nullptr, gamma, pc, lX, 0.f, 0.f, J, dJ, L, q, stream);
}

extern "C" int mi3_reg_xij(const float *bi, const float *lambdas, float gamma, float pc, const float *J, float *dJ,
                           uint32_t L, uint32_t q, void *stream) {
    return launch_reg<R_XIJ>("mi3_reg_xij", bi, lambdas, gamma, pc, 0.f, 0.f, 0.f, J, dJ, L, q, stream);
}

extern "C" int mi3_reg_scadx(const float *bi, float gamma, float pc, float s, float r, float a, const float *J,
                             float *dJ, uint32_t L, uint32_t q, void *stream) {
    return launch_reg<R_SCADX>("mi3_reg_scadx", bi, nullptr, gamma, pc, s, r, a, J, dJ, L, q, stream);
}

extern "C" int mi3_reg_expx(const float *bi, float gamma, float pc, float lam, const float *J, float *dJ,
                            uint32_t L, uint32_t q, void *stream) {
    return launch_reg<R_EXPX>("mi3_reg_expx", bi, nullptr, gamma, pc, lam, 0.f, 0.f, J, dJ, L, q, stream);
}

extern "C" int mi3_reg_dde(const float *bi, float gamma, float pc, float lambda, const float *J, float *dJ,
                           uint32_t L, uint32_t q, void *stream) {
    return launch_reg<R_DDE>("mi3_reg_dde", bi, nullptr, gamma, pc, lambda, 0.f, 0.f, J, dJ, L, q, stream);
}

extern "C" int mi3_reg_scaddde(const float *bi, float gamma, float pc, float lambda, float r, const float *J,
                               float *dJ, uint32_t L, uint32_t q, void *stream) {
    return launch_reg<R_SCADDDE>("mi3_reg_scaddde", bi, nullptr, gamma, pc, lambda, r, 0.f, J, dJ, L, q, stream);
}
