/*
 * mi3b200.h -- C ABI of libmi3b200, the B200 (sm_100a) implementation of
 * Mi3-GPU's inference inner loop (Metropolis sweeps, Potts energies,
 * bimarginal counts, Zwanzig-reweighted quasi-Newton coupling update).
 *
 * Conventions
 *   - Every pointer argument is a DEVICE pointer owned by the caller (for
 *     example a PyTorch CUDA tensor), unless the comment says otherwise.
 *   - Every call is asynchronous on the caller's stream (`stream` is a
 *     cudaStream_t passed as void*; NULL means the legacy default stream).
 *   - Every call returns 0 on success and a negative MI3_ERR_* code on a
 *     rejected argument or a launch failure; mi3_last_error() then returns a
 *     thread-local message.  No C++ exception crosses this boundary.
 *   - Array layouts are the reference's (mi3gpu/mcmcGPU.py:173-184):
 *       J, dJ, bi, bi target : (nPairs, q*q) float32, pair order (i<j) row
 *                              major, residue index q*a+b
 *       bicount              : (nPairs, q*q) uint32
 *       seq                  : (SWORDS, buflen) uint32, SWORDS=(L-1)/4+1,
 *                              byte k of word w = site 4w+k, walker-minor
 *       rngstates            : (N, 4) uint32 = {x.s0, x.s1, c.s0, c.s1}, the
 *                              memory image of mwc64xvec2_state_t ('<2u8')
 *       E, weights, Bs       : (N,) float32
 *   - The one layout that differs is the unpacked coupling table used by the
 *     sampler ("Jrows"): L rows of L blocks of q*q floats, each row padded to
 *     mi3_jrows_stride(L, q) floats, diagonal blocks zero.  The reference's
 *     (L*L, q*q) Junpacked is the same table without the row padding.
 *
 * Each entry point names the reference interface it replaces as
 * file:line in the reference tree (mi3gpu/...).
 */
#ifndef MI3B200_H
#define MI3B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MI3_OK 0
#define MI3_ERR_ARG (-1)       /* bad size, null pointer, unsupported shape   */
#define MI3_ERR_CUDA (-2)      /* CUDA runtime / launch error                 */
#define MI3_ERR_ALIGN (-3)     /* pointer not aligned as required             */
#define MI3_ERR_WORKSPACE (-4) /* workspace too small                         */

/* Status word values written by the sampler kernel (int32 in device memory). */
#define MI3_STATUS_OK 0
#define MI3_STATUS_TIMEOUT_FULL 1  /* consumer gave up waiting for a J chunk   */
#define MI3_STATUS_TIMEOUT_EMPTY 2 /* producer gave up waiting for a free slot */
#define MI3_STATUS_BAD_INPUT 3     /* a site index >= L in position_list       */

/* Thread-local message for the last failed call on this host thread. */
const char *mi3_last_error(void);
/* ABI version of this library. */
int mi3_abi_version(void);

/* Test hook for the failure path of the device-side bounded waits: one
 * thread waits on an mbarrier that nothing completes, with the wait routine
 * the sampler and the tensor-core kernels use, and gives up after limit_ns
 * (<= 2 s): *status (int32, zeroed by the caller) becomes
 * MI3_STATUS_TIMEOUT_FULL and *waited_ns (uint64) the time waited.  With
 * abort_after_ns > 0 another warp raises the CTA's abort flag after that
 * time, which ends the wait early.  Nothing faults or hangs: the kernel
 * returns and the context stays usable. */
int mi3_probe_bounded_wait(int32_t *status, uint64_t limit_ns, uint64_t abort_after_ns,
                           unsigned long long *waited_ns, void *stream);

/* ---------------------------------------------------------------- sampler */

/* initRNG2 (mcmc.cl:349-356) as launched by MCMCGPU._initMCMC_RNG
 * (mcmcGPU.py:410-445): walker g, lane v gets the MWC64X stream at distance
 * rng_offset + (2g+v)*walker_span. */
int mi3_init_rng(uint32_t *rngstates, uint32_t nwalkers, uint64_t rng_offset,
                 uint64_t walker_span, void *stream);

/* Floats per row of the unpacked coupling table (see Conventions). */
uint64_t mi3_jrows_stride(uint32_t L, uint32_t q);

/* unpackfV (mcmc.cl:42-65) as launched by MCMCGPU.unpackJ
 * (mcmcGPU.py:393-408), into the padded Jrows layout (diagonal zeroed).
 * Jrows must hold L*mi3_jrows_stride(L,q) floats, 16-byte aligned. */
int mi3_unpack_j(const float *J, float *Jrows, uint32_t L, uint32_t q, void *stream);

/* metropolis + DeltaEnergy (mcmc.cl:360-458) as launched by MCMCGPU.runMCMC
 * (mcmcGPU.py:460-482): nsteps single-site proposals per walker at the
 * shared sites position_list[position_offset + i] (each < L; residues in
 * seqmem must be < q -- the results are undefined otherwise, but no access
 * leaves the caller's buffers).  betas may be NULL (then
 * every walker uses `beta`, the reference's -DBETA macro; with betas given it
 * is the -DTEMPERING build).  nseqs must be a multiple of 128.  *status
 * (int32, device) receives MI3_STATUS_* if an internal bounded wait gave up;
 * the caller zeroes it. */
int mi3_metropolis(const float *Jrows, uint32_t *rngstates, uint32_t position_offset,
                   const uint32_t *position_list, uint32_t nsteps, const float *betas,
                   float beta, uint32_t *seqmem, uint32_t nseqs, uint32_t L, uint32_t q,
                   int32_t *status, void *stream);

/* mi3_metropolis with an explicit tile plan: walkers per CTA (multiple of
 * 32 in [64, 512] dividing nseqs), sites per coupling chunk (multiple of 4,
 * <= L rounded up to 4) and ring stages ([2, 8]); all three 0 = the
 * built-in choice.  Same results for every plan (the plan only changes the
 * schedule).  No counterpart in the reference (its work-group size is a
 * launch parameter, mcmcGPU.py:1140-1163). */
int mi3_metropolis_plan(const float *Jrows, uint32_t *rngstates, uint32_t position_offset,
                        const uint32_t *position_list, uint32_t nsteps, const float *betas,
                        float beta, uint32_t *seqmem, uint32_t nseqs, uint32_t L, uint32_t q,
                        uint32_t walkers_per_cta, uint32_t sites_per_chunk, uint32_t stages,
                        int32_t *status, void *stream);

/* Valid tile plans for a shape, as (walkers_per_cta, sites_per_chunk,
 * stages) triples into plans[3*max] (nullable); returns how many exist. */
uint32_t mi3_metropolis_plans(uint32_t L, uint32_t q, uint32_t nseqs, uint32_t *plans, uint32_t max);

/* Floats of the chunk-tiled coupling layout of mi3_metropolis_skew:
 * L rows, each of ceil((L + 31) / 32) chunks of [q*q cells][32 sites]. */
uint64_t mi3_jtiles_floats(uint32_t L, uint32_t q);

/* unpackfV (mcmc.cl:42-65) as launched by MCMCGPU.unpackJ
 * (mcmcGPU.py:393-408), into the chunk-tiled layout:
 * Jtiles[pos][k][a*q + b][c] = J_{pos,m}(a, b) for site m = 32 k + c,
 * zero for m == pos and for m >= L.  Jtiles: mi3_jtiles_floats(L, q)
 * floats, 16-byte aligned. */
int mi3_unpack_j_tiles(const float *J, float *Jtiles, uint32_t L, uint32_t q, void *stream);

/* metropolis + DeltaEnergy (mcmc.cl:360-458) as launched by MCMCGPU.runMCMC
 * (mcmcGPU.py:460-482), a second kernel design with identical results to
 * mi3_metropolis (same trajectories and RNG states, bit for bit): each
 * warp's walkers run skewed by one site per lane so that the coupling
 * gathers of a warp hit 32 different shared-memory banks; walker
 * sequences are held in registers.  Reads the chunk-tiled couplings of
 * mi3_unpack_j_tiles.  2 <= q <= 21, nseqs a multiple of 32,
 * walkers_per_cta 256, 512 or 768 (the last CTA may be partly filled):
 * L + 31 <= 288 with 512 or 768, L + 31 <= 576 with 256; 0 picks 512 when
 * L allows it, else 256.  Residues >= q in
 * seqmem are clamped to q - 1.  replicas (0 = 1): Jtiles holds that many
 * identical copies of the table, mi3_jtiles_floats(L, q) floats apart, and
 * CTA b reads copy b % replicas (spreads the CTAs' simultaneous reads of
 * one coupling row over more L2 slices).  status: as mi3_metropolis. */
int mi3_metropolis_skew(const float *Jtiles, uint32_t *rngstates, uint32_t position_offset,
                        const uint32_t *position_list, uint32_t nsteps, const float *betas, float beta,
                        uint32_t *seqmem, uint32_t nseqs, uint32_t L, uint32_t q, uint32_t walkers_per_cta,
                        uint32_t replicas, int32_t *status, void *stream);

/* gen_indep (mcmc.cl:170-244) as launched by MCMCGPU.gen_indep
 * (mcmcGPU.py:380-390); cprob is (L, q-1) cumulative probabilities
 * (MCMCGPU.prepare_indep, mcmcGPU.py:375-378). */
int mi3_gen_indep(uint32_t *seqmem, uint32_t buflen, uint32_t nseq, uint32_t *rngstates,
                  const float *cprob, uint32_t L, uint32_t q, void *stream);

/* --------------------------------------------------------------- energies */

/* Bytes of workspace mi3_energies needs for nseq sequences. */
size_t mi3_energies_workspace(uint32_t nseq);

/* getEnergies (mcmc.cl:249-345) as launched by MCMCGPU.calcEnergies
 * (mcmcGPU.py:536-553): E[n] = sum_{i<j} J[pair(i,j)][q*s_i+s_j] for the
 * first nseq sequences of a buffer of row length buflen.  Each site's row
 * of at most 16 couplings per tile is summed in float, rows in double, tiles
 * in 64-bit fixed point (deterministic); rounded once to float.  The
 * workspace (device, >= mi3_energies_workspace(nseq) bytes, 8-byte aligned)
 * is clobbered. */
int mi3_energies(const float *J, const uint32_t *seqmem, uint32_t buflen, uint32_t nseq,
                 float *energies, uint32_t L, uint32_t q, void *workspace, size_t ws_bytes,
                 void *stream);

/* getEnergies (mcmc.cl:249-345) on the tensor cores: per tile of row and
 * column sites a BF16 one-hot GEMM X_I (J_hi + J_lo)_IJ (tcgen05, FP32
 * accumulation in tensor memory) whose epilogue adds, per sequence, the
 * column its own residues select; tiles are combined in 64-bit fixed point
 * as in mi3_energies.  |E - E_exact| <= 2^-15 sum_{i<j} |J(s_i,s_j)| +
 * 2^-24 |E| (hi + lo carries J to 2^-17; FP32 sums of at most 3*128/q
 * terms).  4 <= q <= 32; the workspace holds nseq uint64 (as
 * mi3_energies_workspace).  *status (int32, device, zeroed by the caller)
 * receives MI3_STATUS_TIMEOUT_FULL if a bounded wait gave up.  No
 * counterpart in the reference. */
int mi3_energies_tc(const float *J, const uint32_t *seqmem, uint32_t buflen, uint32_t nseq, float *energies,
                    uint32_t L, uint32_t q, void *workspace, size_t ws_bytes, int32_t *status, void *stream);

/* Capacity of mi3_energies_noalloc, in sequences. */
#define MI3_ENERGIES_NOALLOC_MAX_SEQ (1u << 20)

/* mi3_energies without a workspace argument, for callers that cannot
 * allocate device memory (for example code running during CUDA graph
 * capture, hosts whose device memory belongs to a pool they do not manage,
 * or language bindings without a device allocator).  No counterpart in the
 * reference: it is an addition of this library.  The accumulators live in
 * an array inside the library: 8 MiB on every GPU where the library's
 * kernels are loaded, held until the process exits.  nseq above
 * MI3_ENERGIES_NOALLOC_MAX_SEQ is rejected with MI3_ERR_ARG.  Every call made
 * outside stream capture looks up the array's device address
 * (cudaGetSymbolAddress) for the current device, so a device reset leaves no
 * stale address; a call made during capture reuses the address of the last
 * call made outside capture on that device.  So make one call on each
 * device (nseq = 0 is enough) before capturing, and again after a
 * cudaDeviceReset; a first call under capture returns MI3_ERR_ARG.
 * The call allocates nothing.  All calls share the one array, so calls whose
 * executions overlap on the GPU (other streams, other threads) race and
 * must be serialised by the caller.  Results equal mi3_energies. */
int mi3_energies_noalloc(const float *J, const uint32_t *seqmem, uint32_t buflen, uint32_t nseq,
                         float *energies, uint32_t L, uint32_t q, void *stream);

/* Bytes of workspace mi3_energies_cons needs (256-byte aligned). */
size_t mi3_energies_cons_workspace(uint32_t L, uint32_t q, uint32_t nseq);

/* mi3_energies with the pair work limited to pairs where neither residue is
 * its site's reference residue cons[i] (device, L bytes, e.g. from
 * mi3_site_consensus): the couplings are moved in FP64 to the gauge where
 * row cons[i] and column cons[j] of every pair block are zero (rounded once
 * to float, in the workspace), the removed parts summed as site fields and
 * a constant in FP64.  Same energies as mi3_energies up to that rounding:
 * |E - E_exact| <= 2^-20 * sum_{i<j} |J'(s_i,s_j)|, with |J'| <= 4 max|J|.
 * L*q*8 + 8 <= 200 KiB.  No counterpart in the reference (an addition of
 * this library). */
int mi3_energies_cons(const float *J, const uint32_t *seqmem, uint32_t buflen, uint32_t nseq,
                      float *energies, uint32_t L, uint32_t q, const uint8_t *cons, void *workspace,
                      size_t ws_bytes, void *stream);

/* ------------------------------------------------- equilibration test */

/* The rank correlation test of runMCMC's automatic equilibration
 * (NewtonSteps.py:395-442, scipy.stats.spearmanr on the energies of the
 * latest checkpoint against one and two checkpoints before, p > 0.02) on
 * the device.  Bytes of workspace mi3_rank_average needs (0 < n < 2^23). */
size_t mi3_rank_workspace(uint32_t n);

/* ranks[i] = the average rank (1-based) of x[i] among x[0..n-1], ties
 * sharing the mean of their positions (scipy.stats.rankdata, method
 * 'average').  x finite; workspace 16-byte aligned. */
int mi3_rank_average(const float *x, uint32_t n, float *ranks, void *workspace, size_t ws_bytes, void *stream);

/* Bytes of workspace mi3_rank_corr needs. */
size_t mi3_rank_corr_workspace(void);

/* *r (double, device) = the Pearson correlation of two rank vectors of
 * mi3_rank_average (spearmanr's statistic), summed in FP64 in a fixed
 * order; NaN when either vector is constant (as spearmanr). */
int mi3_rank_corr(const float *ranks_a, const float *ranks_b, uint32_t n, double *r, void *workspace,
                  size_t ws_bytes, void *stream);

/* *flag (int32, device) = 1 when |*r1| < rcrit and |*r2| < rcrit, else 0
 * (NaN gives 0).  With rcrit = t_c / sqrt(n - 2 + t_c^2), t_c the upper 1%
 * point of Student's t with n - 2 degrees of freedom, this is the
 * reference's "p1 > 0.02 and p2 > 0.02".  No counterpart in the reference
 * (it decides on the host). */
int mi3_equil_decide(const double *r1, const double *r2, double rcrit, int32_t *flag, void *stream);

/* ------------------------------------------------------------ bimarginals */

/* countBivariate (mcmc.cl:462-516) as launched by MCMCGPU.calcBicounts
 * (mcmcGPU.py:501-518): exact uint32 pair histograms. */
int mi3_bicounts(const uint32_t *seqmem, uint32_t buflen, uint32_t nseq, uint32_t *bicount,
                 uint32_t L, uint32_t q, void *stream);

/* countBivariate (mcmc.cl:462-516) on the tensor cores: the same exact
 * uint32 counts as mi3_bicounts, computed as FP8 one-hot GEMMs X^T X with
 * tcgen05 MMAs (FP32 accumulation, exact below 2^24 per chunk).  4 <= q <= 32.
 * *status (int32, device, zeroed by the caller) receives
 * MI3_STATUS_TIMEOUT_FULL if a bounded wait for the tensor cores gave up,
 * or MI3_STATUS_TIMEOUT_EMPTY if the operand producers' wait for a free
 * stage did. */
int mi3_bicounts_tc(const uint32_t *seqmem, uint32_t buflen, uint32_t nseq, uint32_t *bicount,
                    uint32_t L, uint32_t q, int32_t *status, void *stream);

/* Launch plan of mi3_bicounts_tc for a shape (host only, no device work):
 * out4 (nullable) = {output tiles, sequence chunks, sequences per chunk,
 * sites per row tile}; returns 1, or 0 outside the kernel's range
 * (L >= 2, 4 <= q <= 32, nseq >= 1).  A chunk holds at most 2^24
 * sequences, so its FP32 sums of 0/1 products are exact integers. */
uint32_t mi3_bicounts_tc_plan(uint32_t L, uint32_t q, uint32_t nseq, uint32_t *out4);

/* bicounts_to_bimarg (mcmc.cl:518-528), MCMCGPU.bicounts_to_bimarg
 * (mcmcGPU.py:520-534). */
int mi3_bicounts_to_bimarg(const uint32_t *bicount, float *bimarg, uint32_t nseq, uint32_t L,
                           uint32_t q, void *stream);

/* Bytes of workspace mi3_weighted_marg needs for nseq sequences:
 * 256 + 8*L*q (padded to 256) + 4 * nPairs * q*q per chunk of up to 65536
 * sequences. */
size_t mi3_weighted_marg_workspace(uint32_t L, uint32_t q, uint32_t nseq);

/* weightedMarg (mcmc.cl:646-718), MCMCGPU.weightedMarg (mcmcGPU.py:634-661):
 * unnormalised bi[pair][q*a+b] = sum_n w_n [s_i=a][s_j=b] for weights >= 0.
 * Reads the seq main layout directly (no transposed copy needed).  Sums are
 * accumulated as integers in fixed point (each weight rounded to 2^-s,
 * s >= 15 - log2(max w)): per chunk of sequences in uint32, then across
 * chunks in uint64 in a fixed order, so the result is deterministic.
 * cons (device, L bytes, nullable): a reference residue per site, for
 * example from mi3_site_consensus.  With it, only pairs where neither site
 * holds its reference residue are histogrammed; the other bins are rebuilt
 * exactly from per-site sums, so the result is bit-identical to the call
 * without cons, and faster when the reference residues are frequent (it is
 * ignored for q > 64 or L*q*4 + L > 160 KiB).  The workspace
 * (>= mi3_weighted_marg_workspace(L,q,nseq) bytes, 256-byte aligned) is
 * clobbered. */
int mi3_weighted_marg(const float *weights, const uint32_t *seqmem, uint32_t buflen,
                      uint32_t nseq, float *bimarg, uint32_t L, uint32_t q, const uint8_t *cons,
                      void *workspace, size_t ws_bytes, void *stream);

/* Bytes of workspace mi3_weighted_marg_tc needs: 256 + 8 * nPairs * q*q. */
size_t mi3_weighted_marg_tc_workspace(uint32_t L, uint32_t q);

/* weightedMarg (mcmc.cl:646-718) on the tensor cores: the same fixed-point
 * weights as mi3_weighted_marg, split into three byte planes, each an
 * integer one-hot GEMM X^T diag(w_p) X (tcgen05.mma.kind::i8, s32
 * accumulators, exact), recombined into 64-bit sums -- bit-identical to
 * mi3_weighted_marg.  4 <= q <= 32.  *status (int32, device, zeroed by the
 * caller) receives MI3_STATUS_TIMEOUT_FULL if a bounded wait for the tensor
 * cores gave up.  No counterpart in the reference (its kernel is the
 * shared-memory histogram). */
int mi3_weighted_marg_tc(const float *weights, const uint32_t *seqmem, uint32_t buflen, uint32_t nseq,
                         float *bimarg, uint32_t L, uint32_t q, void *workspace, size_t ws_bytes,
                         int32_t *status, void *stream);

/* The walkers as the lines of an MSA text file, in the format of the
 * reference's writeSeqs (mi3gpu/utils/seqload.py:378-411, no id field):
 * line n = alpha[residue] for the L sites of walker n, then '\n', so text
 * (device, 16-byte aligned) receives nseq*(L+1) bytes.  alpha is a HOST
 * pointer to nalpha <= 256 characters.  A residue >= nalpha is written as
 * '?' and *status (int32, device, zeroed by the caller) receives
 * MI3_STATUS_BAD_INPUT. */
int mi3_seqs_to_text(const uint32_t *seqmem, uint32_t buflen, uint32_t nseq, uint32_t L,
                     const char *alpha, uint32_t nalpha, uint8_t *text, int32_t *status, void *stream);

/* MSA text lines back into walkers, the translation of the reference's
 * loadSeqs (seqload.py:91-133, 196-246, 259-352): nseq lines of line_len =
 * id_len + L + 1 bytes each (an id field of id_len bytes whose last byte is
 * a space when id_len > 0, the L residues, '\n') from text (device,
 * 16-byte aligned; headers and end-of-file fix-ups are the caller's) into
 * columns [n0, n0+nseq) of seqmem.  alpha: HOST pointer, nalpha <= 255
 * characters; a character maps to its (last) index in alpha.  *first_bad
 * (uint64, device) receives the index of the first malformed line -- no
 * '\n' at its end, no space ending its id field, or a character not in
 * alpha -- or UINT64_MAX; the words of malformed lines are undefined. */
int mi3_text_to_seqs(const uint8_t *text, uint32_t nseq, uint32_t line_len, uint32_t id_len, uint32_t L,
                     const char *alpha, uint32_t nalpha, uint32_t *seqmem, uint32_t buflen, uint32_t n0,
                     uint64_t *first_bad, void *stream);

/* copySubseq (mcmc.cl:99-122), MCMCGPU.copySubseq (mcmcGPU.py:1001-1014):
 * every sequence of the large buffer (SWORDS, nlarge) takes, at each site i
 * with marks[i] != 0 (marks: device, L bytes), the residue of sequence
 * seqind of the small buffer (SWORDS, nsmall). */
int mi3_copy_subseq(const uint32_t *small, uint32_t nsmall, uint32_t seqind, const uint8_t *marks,
                    uint32_t *large, uint32_t nlarge, uint32_t L, void *stream);

/* Bytes of workspace mi3_site_consensus needs: 8*L*q. */
size_t mi3_site_consensus_workspace(uint32_t L, uint32_t q);

/* cons[i] = the most frequent residue at site i among the first nseq
 * sequences (the lowest on ties); L*q*4 + L <= 160 KiB.  No counterpart in
 * the reference: the consensus residues let the pair kernels skip work (see
 * mi3_weighted_marg and mi3_energies_cons). */
int mi3_site_consensus(const uint32_t *seqmem, uint32_t buflen, uint32_t nseq, uint32_t L, uint32_t q,
                       uint8_t *cons, void *workspace, size_t ws_bytes, void *stream);

/* renormalize_bimarg (mcmc.cl:753-759), MCMCGPU.renormalize_bimarg
 * (mcmcGPU.py:663-668), same summation tree as the reference. */
int mi3_renormalize_bimarg(float *bimarg, uint32_t L, uint32_t q, void *stream);

/* unpackseqs1T (mcmc.cl:124-168), MCMCGPU.repackseqs_T (mcmcGPU.py:356-373):
 * (SWORDS, buf4len) words -> (L, buf1len) words, 4 walkers per word. */
int mi3_repack_seqs_T(const uint32_t *seq4, uint32_t buf4len, uint32_t *seqL, uint32_t buf1len,
                      uint32_t L, void *stream);

/* ------------------------------------------------------ quasi-Newton step */

/* updatedJ (mcmc.cl:829-843), MCMCGPU.updateJ (mcmcGPU.py:704-718):
 * Jo = Ji - gamma*(bi_target - bi)/(bi + pc).  Ji may equal Jo. */
int mi3_update_j(const float *bi_target, const float *bi, float gamma, float pc, const float *Ji,
                 float *Jo, uint32_t L, uint32_t q, void *stream);

/* reg_l1z (mcmc.cl:845-872), MCMCGPU.reg_l1z (mcmcGPU.py:720-731). */
int mi3_reg_l1z(const float *bi, float gamma, float pc, float lJ, const float *J, float *dJ,
                uint32_t L, uint32_t q, void *stream);

/* reg_l2z (mcmc.cl:874-902), MCMCGPU.reg_l2z (mcmcGPU.py:733-745). */
int mi3_reg_l2z(const float *bi, float gamma, float pc, float lJ, const float *J, float *dJ,
                uint32_t L, uint32_t q, void *stream);

/* The other regularizers, each one kernel of mcmc.cl applied per q*q pair
 * block to dJ (in place), with J the current couplings and bi the current
 * bimarginals; 2 <= q <= 32.  Host wrappers in mcmcGPU.py:747-843. */
/* reg_SCADJ (mcmc.cl:904-934): SCAD penalty on the zero-gauge J+dJ. */
int mi3_reg_scadj(const float *bi, float gamma, float pc, float lJ, float a, const float *J, float *dJ,
                  uint32_t L, uint32_t q, void *stream);
/* reg_X (mcmc.cl:1005-1030): penalty on X_ij = sum (J+dJ) C_ij. */
int mi3_reg_x(const float *bi, float lX, float gamma, float pc, const float *J, float *dJ, uint32_t L,
              uint32_t q, void *stream);
/* reg_Xij (mcmc.cl:975-1003): as reg_X with one lambda per pair
 * (lambdas: nPairs floats, the 'Xlambdas' buffer). */
int mi3_reg_xij(const float *bi, const float *lambdas, float gamma, float pc, const float *J, float *dJ,
                uint32_t L, uint32_t q, void *stream);
/* reg_SCADX (mcmc.cl:1078-1121). */
int mi3_reg_scadx(const float *bi, float gamma, float pc, float s, float r, float a, const float *J,
                  float *dJ, uint32_t L, uint32_t q, void *stream);
/* reg_expX (mcmc.cl:1123-1150). */
int mi3_reg_expx(const float *bi, float gamma, float pc, float lam, const float *J, float *dJ, uint32_t L,
                 uint32_t q, void *stream);
/* reg_ddE (mcmc.cl:1152-1188). */
int mi3_reg_dde(const float *bi, float gamma, float pc, float lambda, const float *J, float *dJ,
                uint32_t L, uint32_t q, void *stream);
/* reg_SCADddE (mcmc.cl:1192-1243). */
int mi3_reg_scaddde(const float *bi, float gamma, float pc, float lambda, float r, const float *J,
                    float *dJ, uint32_t L, uint32_t q, void *stream);

/* minFloats (mcmc.cl:558-584), MCMCGPU.min_buf (mcmcGPU.py:555-567):
 * *out = min(0, min(data)) (the reference's accumulator starts at 0). */
int mi3_min_floats(const float *data, uint32_t len, float *out, void *stream);

/* dE_to_weights (mcmc.cl:624-633), MCMCGPU.dE_to_weights (mcmcGPU.py:591-610):
 * w = exp(-dE + ref_E). */
int mi3_dE_to_weights(float ref_E, const float *dE, float *weights, uint32_t n, void *stream);

/* fixed_beta_weights (mcmc.cl:635-644), MCMCGPU.fixed_beta_weights
 * (mcmcGPU.py:613-632): w = exp((beta-1)*(E - ref_E)). */
int mi3_fixed_beta_weights(float beta, float ref_E, const float *E, float *weights, uint32_t n,
                           void *stream);

/* Bytes of workspace mi3_weight_stats / mi3_weights_fused need. */
size_t mi3_weight_stats_workspace(uint32_t n);

/* weight_stats (mcmc.cl:586-622), MCMCGPU.weight_statistics
 * (mcmcGPU.py:569-589): out2 = {sum w, sum w^2} as float; out2_f64 (may be
 * NULL) receives the same sums in double.  Deterministic. */
int mi3_weight_stats(const float *weights, uint32_t n, float *out2, double *out2_f64,
                     void *workspace, size_t ws_bytes, void *stream);

/* One pass of the Newton step's per-sequence work (NewtonSteps.py:226-231):
 * weights = exp(-dE + ref_E), *minout = min(0, min dE), stats = {sum w,
 * sum w^2} (float and double). */
int mi3_weights_fused(float ref_E, const float *dE, float *weights, uint32_t n, float *minout,
                      float *out2, double *out2_f64, void *workspace, size_t ws_bytes,
                      void *stream);

/* ------------------------------------------------ learned proposal (MADE)
 * No counterpart in the reference: a masked autoregressive network over
 * L sites x q residues (two hidden layers of H units) trained on sampled
 * sequences and used as an independence Metropolis-Hastings proposal.
 * Layouts: W1T [Lq][H], b1 [H], W2 [H][H], b2 [H], W3 [Lq][H], b3 [Lq];
 * masked entries are zero and stay zero.  Sequences in the seq layout. */

/* Teacher-forced forward of sequences n0..n0+B-1: h1 = b1 + sum_i W1T[s_i],
 * a1 = relu(h1), h2 = a1 W2^T + b2, a2 = relu(h2), logits = a2 W3^T + b3;
 * logq (nullable) = sum_i log softmax(logits_i)[s_i]. */
int mi3_made_forward(const uint32_t *seq, uint32_t buflen, uint32_t n0, uint32_t B, uint32_t L,
                     uint32_t q, uint32_t H, const float *W1T, const float *b1, const float *W2,
                     const float *b2, const float *W3, const float *b3, float *h1, float *a1, float *h2,
                     float *a2, float *logits, float *logq, void *stream);

/* Gradients of the batch-mean negative log-likelihood (masked), from the
 * forward's activations; dlogits, X (B x Lq), dh1, dh2 (B x H) are scratch;
 * loss_per_seq (nullable) receives log q per sequence. */
int mi3_made_backward(const uint32_t *seq, uint32_t buflen, uint32_t n0, uint32_t B, uint32_t L,
                      uint32_t q, uint32_t H, const float *W2, const float *W3, const float *h1,
                      const float *a1, const float *h2, const float *a2, const float *logits,
                      float *dlogits, float *X, float *dh1, float *dh2, float *gW1T, float *gb1,
                      float *gW2, float *gb2, float *gW3, float *gb3, const float *mW1T,
                      const float *mW2, const float *mW3, float *loss_per_seq, void *stream);

/* The same forward and backward with their dense products as BF16
 * tensor-core GEMMs (mi3_gemm_bf16: operands rounded to bf16, FP32
 * accumulation); workspace of mi3_made_gemm_workspace(B, L, q, H) bytes,
 * 1024-byte aligned; a timed-out wait sets *status. */
uint64_t mi3_made_gemm_workspace(uint32_t B, uint32_t L, uint32_t q, uint32_t H);
int mi3_made_forward_tc(const uint32_t *seq, uint32_t buflen, uint32_t n0, uint32_t B, uint32_t L,
                        uint32_t q, uint32_t H, const float *W1T, const float *b1, const float *W2,
                        const float *b2, const float *W3, const float *b3, float *h1, float *a1, float *h2,
                        float *a2, float *logits, float *logq, void *workspace, uint64_t ws_bytes,
                        int32_t *status, void *stream);
int mi3_made_backward_tc(const uint32_t *seq, uint32_t buflen, uint32_t n0, uint32_t B, uint32_t L,
                         uint32_t q, uint32_t H, const float *W2, const float *W3, const float *h1,
                         const float *a1, const float *h2, const float *a2, const float *logits,
                         float *dlogits, float *X, float *dh1, float *dh2, float *gW1T, float *gb1,
                         float *gW2, float *gb2, float *gW3, float *gb3, const float *mW1T,
                         const float *mW2, const float *mW3, float *loss_per_seq, void *workspace,
                         uint64_t ws_bytes, int32_t *status, void *stream);

/* C (M x N, row stride ldc, FP32) = alpha A B^T + beta C on the tcgen05
 * tensor cores, A(m, k) = A[m sam + k sak], B^T(k, n) = B[k sbk + n sbn]
 * given in FP32 and rounded to bf16, FP32 accumulation.  The operands are
 * packed into workspace (mi3_gemm_bf16_workspace bytes, 1024-byte
 * aligned) first; a timed-out wait sets *status. */
uint64_t mi3_gemm_bf16_workspace(uint32_t M, uint32_t N, uint32_t K);
int mi3_gemm_bf16(uint32_t M, uint32_t N, uint32_t K, const float *A, int64_t sam, int64_t sak,
                  const float *B, int64_t sbk, int64_t sbn, float *C, int64_t ldc, float alpha, float beta,
                  void *workspace, uint64_t ws_bytes, int32_t *status, void *stream);

/* Adam step (bias-corrected, step >= 1) on n parameters p with gradient g
 * and moments m, v; refreshes the bf16-rounded float copy pc and the bf16
 * copy ph (nullable); entries with mask 0 (mask nullable) stay 0. */
int mi3_made_adam(float *p, float *pc, void *ph_bf16, const float *g, float *m, float *v,
                  const float *mask, uint64_t n, float lr, float beta1, float beta2, float eps,
                  uint32_t step, void *stream);

/* pc = bf16-rounded p (as float), ph = the bf16 values (nullable). */
int mi3_made_round_bf16(const float *p, float *pc, void *ph_bf16, uint64_t n, void *stream);

/* Autoregressive sampling of nseq sequences into seq (given = 0), or log q
 * of the sequences in seq (given = 1); hidden-2 units grouped by MADE degree
 * (deg2_start [L+1], deg2_units [H]); one forward pass per sequence.
 * q <= 32, H <= 1024.  Weights in bf16. */
int mi3_made_sample(uint32_t L, uint32_t q, uint32_t H, const void *W1T_bf16, const float *b1,
                    const void *W2_bf16, const float *b2, const void *W3_bf16, const float *b3,
                    const int32_t *deg2_start, const int32_t *deg2_units, uint32_t *seq,
                    uint32_t buflen, uint32_t nseq, float *logq, uint64_t seed, int32_t given,
                    void *stream);

/* Tensor-core MADE sampler (tcgen05).  Hidden degrees m1, m2 (host arrays
 * of H int32, sorted, in [1, L-1]) grouped in blocks of G sites: block b
 * owns the units of degree in (bG, bG+G], 0, 16, 32 or 48 per layer;
 * q in {4, 8}, H <= 512 a multiple of 16, G in {4, 8} with G q <= 32
 * and ceil(L/G) * roundup(G q, 16) + 48 + ceil(L/4) <= 512.  The activations entering
 * layers 2 and 3 are rounded to bf16.
 * mi3_made_tc_workspace: device bytes for the plan's tables and weight
 * tiles (0 if the degrees or sizes are not supported). */
uint64_t mi3_made_tc_workspace(uint32_t L, uint32_t q, uint32_t H, uint32_t G, const int32_t *m1,
                               const int32_t *m2);

/* Build the plan from float weights holding bf16 values (the layouts
 * above) into workspace (256-byte aligned); plan_out (host, 24 uint64)
 * receives the launch parameters.  Call again after the weights change. */
int mi3_made_tc_prepare(uint32_t L, uint32_t q, uint32_t H, uint32_t G, const int32_t *m1,
                        const int32_t *m2, const float *W1T, const float *b1, const float *W2,
                        const float *b2, const float *W3, const float *b3, void *workspace,
                        uint64_t ws_bytes, uint64_t *plan_out, void *stream);

/* Draw nseq sequences into seq (given = 0; residue i of walker n from the
 * uniform (seed, n, i) of mi3_made_sample), or log q of the sequences in
 * seq (given = 1); log q of a drawn sequence is reproduced exactly.  A
 * timed-out wait sets *status (int32, device). */
int mi3_made_tc_sample(const uint64_t *plan, uint32_t *seq, uint32_t buflen, uint32_t nseq,
                       float *logq, uint64_t seed, int32_t given, int32_t *status, void *stream);

/* Independence Metropolis-Hastings: walker n takes proposal n with
 * probability min(1, exp(-(Ep-E)) exp(logq - logq_prop)); accepted walkers
 * copy sequence, energy and log q; *naccept (uint64) += acceptances. */
int mi3_mh_independence(uint32_t *seq, const uint32_t *prop, uint32_t buflen, uint32_t nseq,
                        uint32_t L, float *E, const float *Ep, float *logq, const float *logq_prop,
                        uint64_t seed, unsigned long long *naccept, void *stream);

/* addFloatBufs (mcmc.cl:720-727), MCMCGPU.addFloatBuf (mcmcGPU.py:670-685). */
int mi3_add_float_bufs(float *dst, const float *src, uint32_t n, void *stream);

/* ---- per-round host work on the device (FP64) ---------------------------
 * The reference runs these on the host in numpy each round
 * (NewtonSteps.py:618 fieldlessGaugeEven before sampling; :33-54
 * bimarg_stats / printstats after it); the device forms keep J resident. */

/* Bytes of workspace mi3_gauge_fieldless_even needs: 8*(nPairs*(2q+1) + L*q). */
size_t mi3_gauge_workspace(uint32_t L, uint32_t q);

/* Jout = fieldlessGaugeEven(0, J)[1] (changeGauge.py:37-155: zero gauge with
 * the fields folded evenly into the couplings) computed in FP64 and rounded
 * once to float; Jout may equal J.  J, Jout: nPairs x q*q floats. */
int mi3_gauge_fieldless_even(const float *J, float *Jout, uint32_t L, uint32_t q, void *workspace,
                             size_t ws_bytes, void *stream);

/* Bytes of workspace mi3_bimarg_stats needs: 48 * nPairs. */
size_t mi3_bimarg_stats_workspace(uint32_t L);

/* bimarg_stats + the X statistic of printstats (NewtonSteps.py:33-54) in
 * FP64 into out[6] (device, 8-byte aligned): SSR = sum (t-m)^2, max |t-m|,
 * mean |t-m|/t over entries with t > 0.01f, the number of those entries,
 * X_model = sum J (m - m_a m_b), X_target = sum J (t - t_a t_b) (m_a, m_b the
 * pair's row and column sums).  J may be NULL (then out[4] = out[5] = 0).
 * Deterministic (fixed reduction order). */
int mi3_bimarg_stats(const float *target, const float *model, const float *J, uint32_t L, uint32_t q,
                     double *out, void *workspace, size_t ws_bytes, void *stream);

/* mi3_weights_fused with the reference energy read from device memory
 * (*ref_dev, which must not alias minout): lets a captured Newton loop carry
 * the previous step's min(0, dE) without a host round trip. */
int mi3_weights_fused_dev(const float *ref_dev, const float *dE, float *weights, uint32_t n, float *minout,
                          float *out2, double *out2_f64, void *workspace, size_t ws_bytes, void *stream);

/* ---- whole rounds as CUDA graphs ---------------------------------------
 * No counterpart in the reference (its round loop is host Python,
 * NewtonSteps.py:610-767).  Capture is in relaxed mode; graphs and execs
 * are opaque cudaGraph_t / cudaGraphExec_t handles. */
int mi3_capture_begin(void *stream);
int mi3_capture_end(void *stream, void **graph_out);
int mi3_graph_instantiate(void *graph, void **exec_out);
int mi3_graph_launch(void *exec, void *stream);
int mi3_graph_destroy(void *graph, void *exec);

/* Add a conditional WHILE node at the capture position of `stream` (its
 * condition is 1 at every launch) and start capturing the loop body on
 * body_stream; *handle_out is the condition handle for mi3_newton_control. */
int mi3_capture_while_begin(void *stream, void *body_stream, unsigned long long *handle_out);
/* End the body capture begun by mi3_capture_while_begin. */
int mi3_capture_while_end(void *body_stream);

/* A conditional handle of the graph `stream` is capturing into, reset to
 * `value` (0 or 1) at every launch.  No counterpart in the reference. */
int mi3_cond_handle_create(void *stream, uint32_t value, unsigned long long *handle_out);

/* At the current capture position of `stream`, a conditional IF node on
 * `handle`: its body (captured on body_stream until mi3_capture_if_end)
 * runs once when the handle is non-zero at that point of the launch. */
int mi3_capture_if_begin(void *stream, void *body_stream, unsigned long long handle);
int mi3_capture_if_end(void *body_stream);

/* One checkpoint of runMCMC's automatic equilibration (NewtonSteps.py:
 * 395-442) inside a graph: with test set, equilibrated when |*r1| and
 * |*r2| (Spearman r against one and two checkpoints back, from
 * mi3_rank_corr) are below rcrit (p > 0.02) and calls >= min_equil; the
 * next checkpoint's IF handle (has_next) is set to 1 unless equilibrated
 * or calls >= max_equil.  out (uint32 x 2, device) = {calls, verdict: 1
 * equilibrated, 2 stopped at max_equil, 0 going on}. */
int mi3_equil_control(unsigned long long next, int32_t has_next, const double *r1, const double *r2,
                      double rcrit, int32_t test, uint32_t calls, uint32_t min_equil, uint32_t max_equil,
                      uint32_t *out, void *stream);

/* End-of-step control of a captured Newton loop (NewtonSteps.py:234-246):
 * ++*count; *ref = *minout (the next step's reference energy); the loop
 * continues while Neff = s^2/s2 (wstats64 = {s, s2}) >= neff_min and
 * *count < *max_steps (device word), and stops on non-finite or zero sums
 * (*stopped, if given, becomes 1 at a normal stop and 2 on divergence). */
int mi3_newton_control(unsigned long long handle, const double *wstats64, const float *minout, float *ref,
                       uint32_t *count, const uint32_t *max_steps, double neff_min, uint32_t *stopped,
                       void *stream);

/* The round-to-round Newton budget of MCMCstep (NewtonSteps.py:664-683) on
 * the device.  after = 0 (before the loop): *budget -= 1.5*delta (not below
 * delta) when stats[0] (this round's SSR) > (state[0] + state[1]) / 2, then
 * state = {SSR, min(state[1], SSR)} (state[0] = NaN before the first round).
 * after = 1: *budget = min(2048, (*count - 1) + delta). */
int mi3_newton_adapt(uint32_t after, const double *stats, const uint32_t *count, uint32_t *budget,
                     double *state, uint32_t delta, void *stream);

/* A new non-blocking stream of the current device / its destruction (capture
 * needs streams that no other part of the process uses). */
int mi3_stream_create(void **stream_out);
int mi3_stream_destroy(void *stream);

/* cudaMemsetAsync, for callers without a runtime binding (graph memset nodes). */
int mi3_memset(void *ptr, int value, size_t nbytes, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* MI3B200_H */
