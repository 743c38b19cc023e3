/*
 * mi3_oracle.c -- CPU restatement of Mi3-GPU's inference inner loop.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle for the CUDA
 * library in mi3gpu_b200/csrc.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load it, and only as
 * the checker (or the timed CPU port), never as a product code path.
 *
 * Every function restates one kernel of the reference's OpenCL program
 * (mi3gpu/mcmc.cl) or one host routine of mi3gpu/mcmcGPU.py, following the
 * reference's arithmetic order where the result is floating point, so that a
 * GPU result can be compared bit for bit or within a stated tolerance.  The
 * MWC64X generator (mi3gpu/mwc64x/cl/mwc64x/*.cl, BSD, David Thomas) is
 * restated from its published algorithm: a multiply-with-carry generator with
 * multiplier A=4294883355, modulus M=A*2^32-1 and stream skipping by modular
 * exponentiation.  The restatement is pinned against the reference's own .cl
 * source compiled as C++ (oracle/ref_rng_shim.cpp, built into oracle/_ref).
 *
 * Build: gcc -O2 -ffp-contract=off -fPIC -shared (see oracle/Makefile).
 * Floating point: float arithmetic only where the reference uses float, no
 * contraction, so results match a strict IEEE float evaluation of mcmc.cl.
 */
#include <stdint.h>
#include <stddef.h>
#include <math.h>
#include <string.h>
#include <stdlib.h>

#define MWC_A 4294883355ULL
#define MWC_M 18446383549859758079ULL
#define MWC_BASEID 4077358422479273989ULL

typedef unsigned __int128 u128;

/* (a*b) mod M; equals MWC_MulMod64 (skip_mwc.cl:24-33) for a,b < 2^64, b<M. */
static uint64_t mulmod64(uint64_t a, uint64_t b) {
    return (uint64_t)(((u128)a * (u128)b) % (u128)MWC_M);
}

/* a^e mod M, square and multiply; skip_mwc.cl:39-48. */
static uint64_t powmod64(uint64_t a, uint64_t e) {
    uint64_t acc = 1, sqr = a;
    while (e) {
        if (e & 1) acc = mulmod64(acc, sqr);
        sqr = mulmod64(sqr, sqr);
        e >>= 1;
    }
    return acc;
}

/* Stream seed for element vecOffset of generator gid; skip_mwc.cl:58-76.
 * out[0]=x, out[1]=c. */
void mi3o_mwc_seed(uint64_t gid, uint32_t vecsize, uint32_t vecoffset,
                   uint64_t base, uint64_t gap, uint32_t *x, uint32_t *c) {
    uint64_t dist = base + (gid * vecsize + vecoffset) * gap;  /* wraps mod 2^64 */
    uint64_t m = powmod64(MWC_A, dist);
    uint64_t v = mulmod64(MWC_BASEID, m);
    *x = (uint32_t)(v / MWC_A);
    *c = (uint32_t)(v % MWC_A);
}

/* Skip `dist` steps of one MWC64X lane; skip_mwc.cl:50-56. */
void mi3o_mwc_skip(uint32_t *x, uint32_t *c, uint64_t dist) {
    uint64_t m = powmod64(MWC_A, dist);
    uint64_t v = (uint64_t)(*x) * MWC_A + (uint64_t)(*c);
    v = mulmod64(v, m);
    *x = (uint32_t)(v / MWC_A);
    *c = (uint32_t)(v % MWC_A);
}

/* One MWC step of one lane; mwc64x_rng.cl:17-27 / mwc64xvec2_rng.cl:17-29. */
static inline void mwc_step(uint32_t *x, uint32_t *c) {
    uint32_t X = *x, C = *c;
    uint32_t Xn = (uint32_t)MWC_A * X + C;
    uint32_t carry = (Xn < C) ? 1u : 0u;
    uint32_t Cn = (uint32_t)(((uint64_t)MWC_A * X) >> 32) + carry;
    *x = Xn;
    *c = Cn;
}

/* State layout per walker: uint32[4] = {x.s0, x.s1, c.s0, c.s1}, the memory
 * image of mwc64xvec2_state_t (mwc64xvec2_rng.cl:12). */
static inline void vec2_next(uint32_t *st, uint32_t *r0, uint32_t *r1) {
    *r0 = st[0] ^ st[2];
    *r1 = st[1] ^ st[3];
    mwc_step(&st[0], &st[2]);
    mwc_step(&st[1], &st[3]);
}

void mi3o_vec2_next(uint32_t *st, uint32_t *r0, uint32_t *r1) { vec2_next(st, r0, r1); }

/* initRNG2 (mcmc.cl:349-356): MWC64XVEC2_SeedStreams(offset, span) per walker. */
void mi3o_init_rng(uint32_t *states, uint32_t n, uint64_t offset, uint64_t span) {
    for (uint32_t g = 0; g < n; g++) {
        mi3o_mwc_seed(g, 2, 0, offset, span, &states[4*g+0], &states[4*g+2]);
        mi3o_mwc_seed(g, 2, 1, offset, span, &states[4*g+1], &states[4*g+3]);
    }
}

/* uniformMap (mcmc.cl:29-31). */
static inline float uniform_map(uint32_t i) {
    return (float)(i >> 8) * 0x1.0p-24f;
}

/* Metropolis acceptance exp(x) > u (mcmc.cl:449), with exp rounded correctly
 * to float: the float nearest the exact exponential, obtained from the double
 * exp.  The GPU library makes the same decision. */
int mi3o_accept(float x, float u) {
    if (x >= 0.0f) return 1;
    float e = (float)exp((double)x);
    return e > u;
}

/* unpackfV (mcmc.cl:42-65) into the library's padded row layout:
 * Ju[i*rowstride + j*q*q + a*q + b] = J_ij(a,b), with the (j,i) block the
 * transpose and the diagonal blocks set to zero.  rowstride >= L*q*q. */
void mi3o_unpack_j(const float *J, float *Ju, uint32_t L, uint32_t q, uint64_t rowstride) {
    uint32_t qq = q*q;
    memset(Ju, 0, sizeof(float)*rowstride*L);
    uint64_t n = 0;
    for (uint32_t i = 0; i < L-1; i++) {
        for (uint32_t j = i+1; j < L; j++, n++) {
            for (uint32_t li = 0; li < qq; li++) {
                Ju[(uint64_t)i*rowstride + (uint64_t)j*qq + li] = J[n*qq + li];
                Ju[(uint64_t)j*rowstride + (uint64_t)i*qq + li] = J[n*qq + q*(li%q) + li/q];
            }
        }
    }
}

static inline uint32_t getbyte(uint32_t w, uint32_t k) { return (w >> (8*k)) & 0xffu; }
static inline uint32_t setbyte(uint32_t w, uint32_t k, uint32_t v) {
    return (w & ~(0xffu << (8*k))) | ((v & 0xffu) << (8*k));
}

/* metropolis + DeltaEnergy (mcmc.cl:360-458), one walker after another.
 * seqmem is (SWORDS, nseqs) uint32, 4 sites per word, walker-minor.
 * Ju is the padded unpacked J (mi3o_unpack_j).  betas may be NULL (then
 * `beta` is used for every walker, the -DBETA macro). */
void mi3o_metropolis(const float *Ju, uint64_t rowstride, uint32_t *states,
                     uint32_t position_offset, const uint32_t *position_list,
                     uint32_t nsteps, const float *betas, float beta,
                     uint32_t *seqmem, uint32_t nseqs, uint32_t L, uint32_t q,
                     uint32_t g0, uint32_t g1) {
    uint32_t qq = q*q;
    for (uint32_t g = g0; g < g1; g++) {
        uint32_t *st = &states[4*g];
        float B = betas ? betas[g] : beta;
        for (uint32_t i = 0; i < nsteps; i++) {
            uint32_t pos = position_list[i + position_offset];
            uint32_t r0, r1;
            vec2_next(st, &r0, &r1);
            uint32_t mutres = r0 % q;
            uint32_t sbn = seqmem[(pos/4)*nseqs + g];
            uint32_t seqp = getbyte(sbn, pos%4);
            const float *row = Ju + (uint64_t)pos*rowstride;
            float dE = 0.0f;
            for (uint32_t m = 0; m < L; m++) {
                if (m == pos) continue;
                uint32_t seqm = getbyte(seqmem[(m/4)*nseqs + g], m%4);
                float a = row[(uint64_t)m*qq + q*mutres + seqm];
                float b = row[(uint64_t)m*qq + q*seqp + seqm];
                dE += (a - b);
            }
            float x = -B*dE;
            if (mi3o_accept(x, uniform_map(r1))) {
                sbn = setbyte(sbn, pos%4, mutres);
                seqmem[(pos/4)*nseqs + g] = sbn;
            }
        }
    }
}

/* getEnergiesf (mcmc.cl:249-336): Kahan-compensated float sum over pairs in
 * order (n ascending, m ascending). */
void mi3o_energies_kahan(const float *J, const uint32_t *seqmem, uint32_t buflen,
                         uint32_t nseq, float *E, uint32_t L, uint32_t q) {
    uint32_t qq = q*q;
    for (uint32_t g = 0; g < nseq; g++) {
        float energy = 0.0f, rem = 0.0f;
        uint64_t pair = 0;
        for (uint32_t n = 0; n < L-1; n++) {
            uint32_t sn = getbyte(seqmem[(n/4)*buflen + g], n%4);
            for (uint32_t m = n+1; m < L; m++, pair++) {
                uint32_t sm = getbyte(seqmem[(m/4)*buflen + g], m%4);
                float y = J[pair*qq + q*sn + sm] - rem;
                float t = energy + y;
                rem = (t - energy) - y;
                energy = t;
            }
        }
        E[g] = energy;
    }
}

/* Same energies accumulated in double (the FP64 oracle of E_potts,
 * utils/getSeqEnergies.py:38-60). */
void mi3o_energies_f64(const float *J, const uint32_t *seqmem, uint32_t buflen,
                       uint32_t nseq, double *E, uint32_t L, uint32_t q) {
    uint32_t qq = q*q;
    for (uint32_t g = 0; g < nseq; g++) {
        double e = 0.0;
        uint64_t pair = 0;
        for (uint32_t n = 0; n < L-1; n++) {
            uint32_t sn = getbyte(seqmem[(n/4)*buflen + g], n%4);
            for (uint32_t m = n+1; m < L; m++, pair++) {
                uint32_t sm = getbyte(seqmem[(m/4)*buflen + g], m%4);
                e += (double)J[pair*qq + q*sn + sm];
            }
        }
        E[g] = e;
    }
}

/* countBivariate (mcmc.cl:462-516): bicount[pair][q*si+sj] over nseq seqs. */
void mi3o_count_bivariate(const uint32_t *seqmem, uint32_t buflen, uint32_t nseq,
                          uint32_t *bicount, uint32_t L, uint32_t q) {
    uint32_t qq = q*q;
    uint64_t npairs = (uint64_t)L*(L-1)/2;
    memset(bicount, 0, sizeof(uint32_t)*npairs*qq);
    uint8_t *s = (uint8_t*)malloc(L);
    for (uint32_t g = 0; g < nseq; g++) {
        for (uint32_t i = 0; i < L; i++) s[i] = (uint8_t)getbyte(seqmem[(i/4)*buflen + g], i%4);
        uint64_t pair = 0;
        for (uint32_t i = 0; i < L-1; i++)
            for (uint32_t j = i+1; j < L; j++, pair++)
                bicount[pair*qq + q*s[i] + s[j]]++;
    }
    free(s);
}

/* bicounts_to_bimarg (mcmc.cl:518-528). */
void mi3o_bicounts_to_bimarg(const uint32_t *bicount, float *bimarg, uint32_t nseq, uint64_t n) {
    for (uint64_t k = 0; k < n; k++) bimarg[k] = ((float)bicount[k]) / ((float)nseq);
}

/* minFloats (mcmc.cl:558-584) with vsize work items: starts each partial at 0,
 * so the result is min(0, min(data)). */
float mi3o_min_floats(const float *data, uint32_t len) {
    float r = 0.0f;
    for (uint32_t n = 0; n < len; n++) r = fminf(data[n], r);
    return r;
}

/* weight_stats (mcmc.cl:586-622) with vsize=1024 work items: strided float
 * partials, then a power-of-two tree. */
void mi3o_weight_stats(const float *data, uint32_t len, float *out2) {
    enum { V = 1024 };
    static float s[V], s2[V];
    for (uint32_t li = 0; li < V; li++) {
        s[li] = 0.0f; s2[li] = 0.0f;
        for (uint32_t n = li; n < len; n += V) {
            float v = data[n];
            s[li] += v;
            s2[li] += v*v;
        }
    }
    for (uint32_t m = V/2; m > 0; m >>= 1)
        for (uint32_t li = 0; li < m; li++) { s[li] = s[li] + s[li+m]; s2[li] = s2[li] + s2[li+m]; }
    out2[0] = s[0]; out2[1] = s2[0];
}

/* Σw and Σw² in double, the FP64 statistic the library reports. */
void mi3o_weight_stats_f64(const float *data, uint32_t len, double *out2) {
    double a = 0.0, b = 0.0;
    for (uint32_t n = 0; n < len; n++) { double v = data[n]; a += v; b += v*v; }
    out2[0] = a; out2[1] = b;
}

/* dE_to_weights (mcmc.cl:624-633). */
void mi3o_dE_to_weights(float ref_E, const float *dE, float *w, uint32_t n) {
    for (uint32_t k = 0; k < n; k++) w[k] = expf(-dE[k] + ref_E);
}

/* fixed_beta_weights (mcmc.cl:635-644). */
void mi3o_fixed_beta_weights(float beta, float ref_E, const float *E, float *w, uint32_t n) {
    for (uint32_t k = 0; k < n; k++) w[k] = expf((beta - 1.0f)*(E[k] - ref_E));
}

/* weightedMarg (mcmc.cl:646-718), unnormalised, accumulated in double.
 * Input in the seq main layout (SWORDS, buflen). */
void mi3o_weighted_marg_f64(const float *w, const uint32_t *seqmem, uint32_t buflen,
                            uint32_t nseq, double *bi, uint32_t L, uint32_t q) {
    uint32_t qq = q*q;
    uint64_t npairs = (uint64_t)L*(L-1)/2;
    memset(bi, 0, sizeof(double)*npairs*qq);
    uint8_t *s = (uint8_t*)malloc(L);
    for (uint32_t g = 0; g < nseq; g++) {
        for (uint32_t i = 0; i < L; i++) s[i] = (uint8_t)getbyte(seqmem[(i/4)*buflen + g], i%4);
        double wg = w[g];
        uint64_t pair = 0;
        for (uint32_t i = 0; i < L-1; i++)
            for (uint32_t j = i+1; j < L; j++, pair++)
                bi[pair*qq + q*s[i] + s[j]] += wg;
    }
    free(s);
}

/* sumqq (mcmc.cl:732-751): odd-aware tree over the q*q block. */
static float sumqq(const float *v, uint32_t qq) {
    float scratch[1024];
    for (uint32_t li = 0; li < qq; li++) scratch[li] = v[li];
    uint32_t m = qq;
    while (m > 1) {
        uint32_t odd = m % 2;
        m = (m + 1) >> 1;
        for (uint32_t li = 0; li < m - odd; li++) scratch[li] = scratch[li] + scratch[li + m];
    }
    return scratch[0];
}

/* renormalize_bimarg (mcmc.cl:753-759). */
void mi3o_renormalize_bimarg(float *bi, uint64_t npairs, uint32_t q) {
    uint32_t qq = q*q;
    for (uint64_t p = 0; p < npairs; p++) {
        float s = sumqq(bi + p*qq, qq);
        for (uint32_t li = 0; li < qq; li++) bi[p*qq + li] = bi[p*qq + li] / s;
    }
}

/* zeroGauge (mcmc.cl:764-822) on one q*q block, in the reference's tree
 * order; writes the zero-gauge block to J0. */
static void zero_gauge_block(const float *Jb, float *J0, uint32_t q) {
    uint32_t qq = q*q;
    float scratch[1024], hi[32], hj[32];
    uint32_t m, li;
    for (li = 0; li < qq; li++) scratch[li] = Jb[li];
    m = q;
    while (m > 1) {
        uint32_t odd = m % 2;
        m = (m + 1) >> 1;
        for (li = 0; li < qq; li++) if (li % q < m - odd) scratch[li] = scratch[li] + scratch[li + m];
    }
    for (li = 0; li < q; li++) hi[li] = scratch[q*li] / (float)q;
    for (li = 0; li < qq; li++) scratch[q*(li % q) + li/q] = Jb[li];
    m = q;
    while (m > 1) {
        uint32_t odd = m % 2;
        m = (m + 1) >> 1;
        for (li = 0; li < qq; li++) if (li % q < m - odd) scratch[li] = scratch[li] + scratch[li + m];
    }
    for (li = 0; li < q; li++) hj[li] = scratch[q*li] / (float)q;
    m = q;
    while (m > 1) {
        uint32_t odd = m % 2;
        m = (m + 1) >> 1;
        for (li = 0; li < m - odd; li++) scratch[q*li] = scratch[q*li] + scratch[q*(li + m)];
    }
    float mean = scratch[0] / (float)q / (float)q;
    for (li = 0; li < q; li++) { hi[li] = hi[li] - mean; hj[li] = hj[li] - mean; }
    for (li = 0; li < qq; li++) J0[li] = Jb[li] - (hi[li/q] + hj[li%q]) - mean;
}

void mi3o_zero_gauge_block(const float *Jb, float *J0, uint32_t q) { zero_gauge_block(Jb, J0, q); }

static inline float ocl_sign(float x) {
    if (x > 0.0f) return 1.0f;
    if (x < 0.0f) return -1.0f;
    if (x != x) return 0.0f;
    return x;  /* keeps the sign of zero */
}

/* updatedJ (mcmc.cl:829-843). */
void mi3o_updatedJ(const float *bt, const float *bi, float gamma, float pc,
                   const float *Ji, float *Jo, uint64_t n) {
    for (uint64_t k = 0; k < n; k++) Jo[k] = Ji[k] - gamma*(bt[k] - bi[k])/(bi[k] + pc);
}

/* reg_l1z (mcmc.cl:845-872) and reg_l2z (mcmc.cl:874-902). l2 != 0 selects l2z. */
void mi3o_reg_lz(const float *bi, float gamma, float pc, float lJ, const float *J,
                 float *dJ, uint64_t npairs, uint32_t q, int l2) {
    uint32_t qq = q*q;
    float Jt[1024], J0[1024];
    for (uint64_t p = 0; p < npairs; p++) {
        for (uint32_t li = 0; li < qq; li++) Jt[li] = J[p*qq + li] + dJ[p*qq + li];
        zero_gauge_block(Jt, J0, q);
        for (uint32_t li = 0; li < qq; li++) {
            uint64_t n = p*qq + li;
            float Jp = dJ[n];
            float j0 = J0[li];
            float R = l2 ? -lJ*j0*gamma/(bi[n] + pc)
                         : -lJ*ocl_sign(j0)*gamma/(bi[n] + pc);
            if (ocl_sign(j0) != ocl_sign(j0 + R)) Jp = Jp - j0;
            else Jp = Jp + R;
            dJ[n] = Jp;
        }
    }
}

/* gen_indep (mcmc.cl:170-244): independent-site sequences from cumulative
 * probabilities cprob (L, q-1). */
void mi3o_gen_indep(uint32_t *seqmem, uint32_t buflen, uint32_t nseq, uint32_t *states,
                    const float *cprob, uint32_t L, uint32_t q) {
    for (uint32_t g = 0; g < nseq; g++) {
        uint32_t *st = &states[4*g];
        uint32_t r0 = 0, r1 = 0, sbn = 0;
        uint32_t pos;
        for (pos = 0; pos < L; pos++) {
            float r;
            if (pos % 2 == 0) { vec2_next(st, &r0, &r1); r = uniform_map(r0); }
            else r = uniform_map(r1);
            const float *cp = cprob + (uint64_t)pos*(q-1);
            uint32_t bot = 0, mid;
            for (uint32_t span = q; span > 1; span -= mid) {
                mid = span / 2;
                if (r >= cp[bot + mid - 1]) bot += mid;
            }
            sbn = setbyte(sbn, pos % 4, bot);
            if ((pos + 1) % 4 == 0) seqmem[(pos/4)*buflen + g] = sbn;
        }
        if (pos % 4 != 0) {
            for (uint32_t l = pos % 4; l < 4; l++) sbn = setbyte(sbn, l, 0);
            seqmem[(pos/4)*buflen + g] = sbn;
        }
    }
}

/* unpackseqs1T (mcmc.cl:124-168): (SWORDS, n) words -> (L, n) bytes. */
void mi3o_repack_seqs_T(const uint32_t *seq4, uint32_t buf4len, uint8_t *seqL,
                        uint32_t buf1len_bytes, uint32_t L) {
    for (uint32_t i = 0; i < L; i++)
        for (uint32_t n = 0; n < buf4len; n++)
            seqL[(uint64_t)i*buf1len_bytes + n] = (uint8_t)getbyte(seq4[(i/4)*buf4len + n], i%4);
}

/* ---------------------------------------------------------------------------
 * Remaining regularizers (mcmc.cl:904-1243), one q*q block per pair, with
 * the reference's reduction trees and operation order.
 */

/* odd-aware tree over the q columns of each row of a q*q scratch block */
static void rows_tree(float *sc, uint32_t q) {
    uint32_t m = q, qq = q*q;
    while (m > 1) {
        uint32_t odd = m % 2;
        m = (m + 1) >> 1;
        for (uint32_t li = 0; li < qq; li++) if (li % q < m - odd) sc[li] = sc[li] + sc[li + m];
    }
}

/* getUnimarg (mcmc.cl:936-973): row sums fi[a], column sums fj[b] */
static void get_unimarg(const float *fij, float *fi, float *fj, uint32_t q) {
    float sc[1024];
    uint32_t qq = q*q;
    for (uint32_t li = 0; li < qq; li++) sc[li] = fij[li];
    rows_tree(sc, q);
    for (uint32_t a = 0; a < q; a++) fi[a] = sc[q*a];
    for (uint32_t li = 0; li < qq; li++) sc[q*(li % q) + li/q] = fij[li];
    rows_tree(sc, q);
    for (uint32_t b = 0; b < q; b++) fj[b] = sc[q*b];
}

/* getXijab (mcmc.cl:1051-1067) for element li */
static float get_xijab(const float *Jt, const float *fi, const float *fj, uint32_t li, uint32_t q) {
    uint32_t c = li / q, d = li % q;
    float x = 0.0f;
    for (uint32_t a = 0; a < q; a++)
        for (uint32_t b = 0; b < q; b++)
            x += Jt[a*q + b]*(fi[a] - (float)(a == c))*(fj[b] - (float)(b == d));
    return x;
}

/* kind: 0 SCADJ(p0=lJ, p1=a), 1 X(p0=lX), 2 Xij(lambdas), 3 SCADX(p0=s, p1=r, p2=a),
 *       4 expX(p0=lam), 5 ddE(p0=lambda), 6 SCADddE(p0=lambda, p1=r) */
void mi3o_reg_other(int kind, const float *bi, const float *lambdas, float gamma, float pc,
                    float p0, float p1, float p2, const float *J, float *dJ, uint64_t npairs,
                    uint32_t q) {
    uint32_t qq = q*q;
    float Jt[1024], Jp[1024], fij[1024], C[1024], J0[1024], sc[1024], fi[32], fj[32], out[1024];
    for (uint64_t p = 0; p < npairs; p++) {
        for (uint32_t li = 0; li < qq; li++) {
            Jp[li] = dJ[p*qq + li];
            Jt[li] = J[p*qq + li] + Jp[li];
            fij[li] = bi[p*qq + li];
        }
        if (kind == 0) {                                   /* reg_SCADJ :904-934 */
            float lJ = p0, a = p1;
            zero_gauge_block(Jt, J0, q);
            for (uint32_t li = 0; li < qq; li++) {
                float j0 = J0[li], R = 0.0f;
                if (fabsf(j0) < lJ) R = fminf(lJ, fabsf(j0)/gamma);
                else if (fabsf(j0) < a*lJ) R = (a*lJ - fabsf(j0))/(a - 1.0f);
                R *= gamma*ocl_sign(j0)/(fij[li] + pc);
                out[li] = Jp[li] - R;
            }
        } else if (kind <= 4) {                            /* X-based :975-1150 */
            get_unimarg(fij, fi, fj, q);
            for (uint32_t li = 0; li < qq; li++) C[li] = fij[li] - fi[li/q]*fj[li%q];
            for (uint32_t li = 0; li < qq; li++) sc[li] = Jt[li]*C[li];
            float X = sumqq(sc, qq);
            float Xnorm = 0.0f;
            if (kind != 4) {
                for (uint32_t li = 0; li < qq; li++) sc[li] = C[li]*C[li]/(fij[li] + pc);
                Xnorm = sumqq(sc, qq);
            }
            for (uint32_t li = 0; li < qq; li++) {
                float c = C[li], f = fij[li];
                if (kind == 1) {                           /* reg_X :1005-1030 */
                    float lX = fminf(p0, fabsf(X)/(Xnorm*gamma));
                    out[li] = Jp[li] - gamma*lX*c*ocl_sign(X)/(f + pc);
                } else if (kind == 2) {                    /* reg_Xij :975-1003 */
                    float lX = fminf(lambdas[p], fabsf(X)/(Xnorm*gamma));
                    float R = lX*c*ocl_sign(X);
                    out[li] = Jp[li] - gamma*R/(f + pc);
                } else if (kind == 3) {                    /* reg_SCADX :1078-1121 */
                    float s = p0, r = p1, a = p2;
                    float xab = get_xijab(Jt, fi, fj, li, q);
                    float R = 0.0f;
                    if (fabsf(X) < r) {
                        r = fminf(r, fabsf(X)/(Xnorm*gamma*s));
                        R = r*ocl_sign(X);
                    } else if (fabsf(X) < a*r) {
                        R = (a*r*ocl_sign(X) - X)/(a - 1.0f);
                    }
                    R *= gamma*s*(c + f*(X - xab))/(f + pc);
                    out[li] = Jp[li] - R;
                } else {                                   /* reg_expX :1123-1150 */
                    float xab = get_xijab(Jt, fi, fj, li, q);
                    float R = ocl_sign(X)*expf(-fabsf(X)/p0)*(c + f*(X - xab));
                    out[li] = Jp[li] - gamma*R/(f + pc);
                }
            }
        } else {                                           /* ddE :1152-1243 */
            float lambda = p0, r = p1;
            for (uint32_t li = 0; li < qq; li++) {
                uint32_t a = li / q, b = li % q;
                float dR = 0.0f;
                for (uint32_t g = 1; g < q; g++) {
                    float jr = Jt[q*a + b] - Jt[q*((a + g) % q) + b];
                    for (uint32_t d = 1; d < q; d++) {
                        float jc = -Jt[q*a + (b + d) % q] + Jt[q*((a + g) % q) + (b + d) % q];
                        float dde = jr + jc;
                        if (kind == 5) {
                            dR += ocl_sign(dde);
                        } else {
                            float R = 0.0f, absD = fabsf(dde);
                            if (absD < r) R = 1.0f;
                            else if (absD < 4.0f*r) R = (4.0f*r - absD)/(4.0f*r - r);
                            dR += lambda*ocl_sign(dde)*R;
                        }
                    }
                }
                dR = dR / (float)((q - 1)*(q - 1));
                if (kind == 5) out[li] = Jp[li] - lambda*dR*gamma/(fij[li] + pc);
                else out[li] = Jp[li] - gamma*dR/(fij[li] + pc);
            }
        }
        for (uint32_t li = 0; li < qq; li++) dJ[p*qq + li] = out[li];
    }
}
