// made_tc.cu -- autoregressive sampling (and teacher-forced log q) of the
// MADE proposal with the bulk of the network on the tcgen05 tensor cores.
//
// Network (as in made.cu): h1 = b1 + sum_j W1T[(j, s_j)], a1 = bf16(relu(h1)),
// h2 = b2 + W2 a1, a2 = bf16(relu(h2)), logits = b3 + W3 a2, with MADE masks
// (hidden-1 unit v sees sites j < m1[v], hidden-2 unit u sees hidden-1 units
// with m1 <= m2[u], output site i sees hidden-2 units with m2 <= i).  The
// activations entering layers 2 and 3 are rounded to bf16, as the tensor
// cores read them; weights are bf16 values, sums are FP32.
//
// Degree blocks.  The hidden degrees are grouped in blocks of G sites
// (G = 4 or 8, G q <= 32): block b owns the units of degree in
// (bG, bG + G], unit indices sorted by degree, 16, 32 or 48 units per
// block and layer.
// Walking the sites in order, when block b starts (sites < s0 = bG drawn):
//   * every hidden-1 unit of an earlier block is final, so the hidden-2
//     units of block b get their share from them as one GEMM,
//       D2 = A1[:, 0:c1] . W2[U2_b, 0:c1]^T      (tcgen05, D2 in TMEM)
//     where A1 (128 walkers x H, bf16, shared memory) holds the final a1;
//   * the logits of every site of block b already hold the share of all
//     hidden-2 units of earlier blocks: after each block the new units'
//     a2 (128 x n2_b, bf16) are multiplied into a TMEM accumulator of the
//     logits of all later sites (tcgen05, acc3 += A2 . W3[later, U2_b]^T).
// What remains inside a block -- the block's own hidden-1 units (their
// inputs from earlier sites gathered once, then one weight row per drawn
// site), its hidden-2 units (one dot product over the block's hidden-1
// units each, as they become final) and the in-block share of each site's
// logits -- runs on the CUDA cores, two or three threads per walker (one
// per 16 units), from weights staged in shared memory.  Masked weights are zero, so each in-block loop
// runs over all of the block's units.
//
// CTA: 128 walkers (TMEM lanes).  8 or 12 warps run the walkers; the next
// warp issues the MMAs; one streams their weight tiles (pre-swizzled K-major
// images, one 1-D bulk copy each) through a 2-stage ring; one streams the
// CUDA-core weights (the layer-1 rows of the earlier sites in FP32 chunks
// of 64 / q sites, then the block's layer-2 and layer-3 weights and the
// layer-1 rows of its own sites in bf16) through a 2- or 3-stage ring.  Each walker's
// sequence words are kept in spare TMEM columns for the layer-1 gathers.
// All waits are bounded (status word).  The kernel draws walker n's
// residue i from the same counter-based uniform as made.cu (seed, n, i);
// with given = 1 it reads the residues instead and returns log q: the same
// arithmetic, so log q of a drawn sequence is reproduced bit for bit.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "made.cuh"
#include "tc.cuh"

namespace mi3 {

constexpr uint32_t MT_M = 128;        // walkers per tile
constexpr uint32_t MT_NU = 48;        // largest unit count per block and layer
constexpr uint32_t MT_HMAX = 512;     // hidden units (A1 holds 8 K-chunks of 64)
constexpr uint32_t MT_GQMAX = 32;     // sites x residues per block
constexpr uint32_t MT_CROWS = 64;     // layer-1 rows (site, residue) per chunk: 64 / q sites
constexpr uint32_t MT_STAGE_ROWS = 64;
constexpr uint32_t MT_STAGE_BYTES = MT_STAGE_ROWS * 128;
constexpr uint32_t MT_WSTAGE_BYTES = 12288;
constexpr uint32_t MT_ROW_BYTES = MT_NU * 2;  // one bf16 weight row over a block's units
constexpr uint32_t MT_W2_BYTES = MT_NU * MT_ROW_BYTES;
constexpr uint32_t MT_W3_BYTES = MT_GQMAX * MT_ROW_BYTES;
// a block's CUDA-core weights besides the layer-1 prefix: W2 [48][48], W3
// [G q][48] and the layer-1 rows of its own sites [G q][48], bf16
// then the block's small parameters (FP32 b3 [G q], b2 [48], and int32
// cnt [16]: block-local index of the first hidden-2 unit of degree
// >= s0 + 1 + k), so that no global load sits on a site's critical path
constexpr uint32_t MT_PAR_OFF = MT_W2_BYTES + 2 * MT_W3_BYTES;
constexpr uint32_t MT_PAR_B3 = 0, MT_PAR_B2 = MT_GQMAX, MT_PAR_CNT = MT_PAR_B2 + MT_NU;
constexpr uint32_t MT_W123_BYTES = MT_PAR_OFF + (MT_PAR_CNT + 16) * 4;
constexpr uint32_t MT_A1_BYTES = (MT_HMAX / 64) * MT_M * 128;
constexpr uint32_t MT_A2_BYTES = MT_M * 128;
constexpr uint32_t MT_TMEM_COLS = 512;
static_assert(MT_W123_BYTES <= MT_WSTAGE_BYTES && MT_CROWS * MT_NU * 4 <= MT_WSTAGE_BYTES, "weight stage");

// One weight tile of the MMA ring and the MMAs that consume it.
struct MtOp {
    uint32_t off;     // byte offset of the tile image
    uint32_t rows;    // N of the MMA (tile rows, 128 B each)
    uint32_t kc;      // A1 K-chunk (layer-2 tiles)
    uint32_t ksteps;  // K / 16 in this tile
    uint32_t dcol;    // TMEM column of the accumulator
    uint32_t first;   // 1: the first tile of a layer-2 product (overwrite D2)
    uint32_t kind;    // 0: layer-2 prefix, 1: logits accumulator update
    uint32_t blk;
};

// One stage of the CUDA-core weight ring: a layer-1 chunk (FP32 rows (j, a)
// of 64 / q sites x the block's hidden-1 units) or the block's in-block
// weights (bf16).
struct MtWOp {
    uint32_t off, bytes, kind, blk, chunk, pad0, pad1, pad2;
};

__host__ __device__ __forceinline__ uint32_t op_bytes(const MtOp &o) { return o.rows * 128; }
__host__ __device__ __forceinline__ uint32_t op_bytes(const MtWOp &o) { return o.bytes; }

// per block: c1 (hidden-1 units before the block), n1, c2, n2, first op of
// the layer-2 tiles, first op of the logits tiles, end, D2 valid, first
// weight-ring op, layer-1 chunks
constexpr uint32_t MT_BLK = 12;

struct MtPlan {
    uint32_t L, q, H, G, nb, N3, d2col, wcol, nops, nwops, nu, pad;
    uint64_t img_bytes, wimg_bytes;
    const MtOp *ops;
    const MtWOp *wops;
    const uint32_t *blk;
    const int32_t *deg2_start;  // [L + 1]: first hidden-2 unit of degree >= d
    const unsigned char *img;   // MMA weight tiles
    const unsigned char *wimg;  // CUDA-core weight stages
    const float *b1b;           // [nb][NU]
    const float *b2b;           // [nb][NU]
    const float *b3;            // [L q]
};
static_assert(sizeof(MtPlan) <= 24 * 8, "plan blob");

__device__ __forceinline__ uint32_t mt_idesc(uint32_t n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((MT_M >> 4) << 24);
}

__device__ __forceinline__ void mt_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// byte offset of (row, k) in a K-major 128B-swizzled tile of 64 K
__device__ __forceinline__ uint32_t mt_sw(uint32_t row, uint32_t k) {
    return row * 128 + ((((k >> 3) ^ (row & 7)) & 7) << 4) + ((k & 7) << 1);
}

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
    return (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(lo)) |
           ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(hi)) << 16);
}

// 8 bf16 (one 16-byte word) -> floats
__device__ __forceinline__ void unpack8(const uint4 w, float *f) {
    f[0] = __uint_as_float(w.x << 16);
    f[1] = __uint_as_float(w.x & 0xffff0000u);
    f[2] = __uint_as_float(w.y << 16);
    f[3] = __uint_as_float(w.y & 0xffff0000u);
    f[4] = __uint_as_float(w.z << 16);
    f[5] = __uint_as_float(w.z & 0xffff0000u);
    f[6] = __uint_as_float(w.w << 16);
    f[7] = __uint_as_float(w.w & 0xffff0000u);
}


// The FP32 layer-1 rows of a chunk hold their 16-byte groups in the order
// g ^ mt_rsw(row): the 4 (q=4) or 8 (q=8) rows a warp reads for one site
// then fall in different bank groups.
__host__ __device__ __forceinline__ uint32_t mt_rsw(uint32_t row) { return (row >> 1) & 3; }

__device__ __forceinline__ uint32_t tmem_ld1(uint32_t taddr) {
    uint32_t r;
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(r) : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    return r;
}

// single-column TMEM store; the writer waits (tcgen05.wait::st) before it
// reads the column back
__device__ __forceinline__ void tmem_st1(uint32_t taddr, uint32_t v) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x1.b32 [%0], {%1};" ::"r"(taddr), "r"(v) : "memory");
}

__device__ __forceinline__ void tmem_ld4(uint32_t taddr, float (&v)[4]) {
    uint32_t r0, r1, r2, r3;
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    v[0] = __uint_as_float(r0);
    v[1] = __uint_as_float(r1);
    v[2] = __uint_as_float(r2);
    v[3] = __uint_as_float(r3);
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                   "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ void tmem_zero16(uint32_t taddr) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1};" ::"r"(
            taddr),
        "r"(0u)
        : "memory");
}

template <uint32_t Q>
__device__ __forceinline__ void tmem_ldq(uint32_t taddr, float (&v)[Q]);
template <>
__device__ __forceinline__ void tmem_ldq<4>(uint32_t taddr, float (&v)[4]) {
    tmem_ld4(taddr, v);
}
template <>
__device__ __forceinline__ void tmem_ldq<8>(uint32_t taddr, float (&v)[8]) {
    tmem_ld8(taddr, v);
}

// One producer thread: stream a list of records into a ring, once per tile
// this CTA owns; on exit wait for the copies still in flight.
template <typename Op, uint32_t NS, uint32_t SB>
__device__ __forceinline__ void mt_produce(const Op *ops, uint32_t nops, const unsigned char *src, unsigned char *ring,
                                           uint64_t *full, uint64_t *empty, uint32_t ntiles,
                                           volatile int *abort_flag, int32_t *status) {
    uint32_t it = 0;
    bool ok = true;
    for (uint32_t t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
        for (uint32_t o = 0; o < nops; ++o) {
            const uint32_t s = it % NS, round = it / NS;
            if (round > 0 && !mbar_wait_bounded(&empty[s], (round - 1) & 1, abort_flag, WAIT_LIMIT_NS)) {
                report(status, ST_TIMEOUT_EMPTY);
                *abort_flag = 1;
                ok = false;
                break;
            }
            const Op op = ops[o];
            const uint32_t bytes = op_bytes(op);
            mbar_arrive_expect_tx(&full[s], bytes);
            bulk_g2s(ring + s * SB, src + op.off, bytes, &full[s]);
            ++it;
        }
    }
    for (uint32_t k = 0; k < NS && k < it; ++k) {
        const uint32_t j = it - 1 - k;
        mbar_wait_bounded(&full[j % NS], (j / NS) & 1, nullptr, WAIT_LIMIT_NS);
    }
}

// Compute threads: NU / 16 warps per TMEM lane quadrant (32 walkers), warp w
// owning walker 32 (w % 4) + lane and unit slice w / 4 (16 of a block's
// units).  Sums over a block's units are taken per slice and added across
// the slices through shared memory in slice order, so the threads of a
// walker hold identical logits and draw the same residue.
template <uint32_t Q, uint32_t NU>
struct MtShape {
    static constexpr uint32_t SL = NU / 16;           // unit slices
    static constexpr uint32_t CT = SL * MT_M;         // compute threads
    static constexpr uint32_t THREADS = CT + 96;      // + MMA issue, MMA-tile and weight producer warps
    static constexpr uint32_t ST = 2;                 // MMA weight-tile ring stages
    static constexpr uint32_t WST = Q == 4 ? 3 : 2;   // CUDA-core weight ring stages
    static constexpr uint32_t HG = 4;                 // hidden-2 units reduced per barrier
    static constexpr uint32_t RED_LG = 2 * Q * SL * MT_M * 4;
    static constexpr uint32_t RED_H2 = 2 * HG * SL * MT_M * 4;
    static constexpr uint32_t SMEM =
        1024 + MT_A1_BYTES + MT_A2_BYTES + ST * MT_STAGE_BYTES + WST * MT_WSTAGE_BYTES + RED_LG + RED_H2 + 256;
    static_assert(SMEM <= 232448, "shared memory");
};

// sum of a 16-unit slice of a bf16 row in shared memory times x, four partial sums
__device__ __forceinline__ float dot16(const unsigned char *row, const float *x) {
    const uint4 w0 = *reinterpret_cast<const uint4 *>(row), w1 = *reinterpret_cast<const uint4 *>(row + 16);
    float f[16];
    unpack8(w0, f);
    unpack8(w1, f + 8);
    float s[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (uint32_t e = 0; e < 16; ++e) s[e & 3] = __fmaf_rn(f[e], x[e], s[e & 3]);
    return (s[0] + s[1]) + (s[2] + s[3]);
}

// h[k] += row[k], k < 16, for a 16-unit slice of a bf16 row
__device__ __forceinline__ void add16h(const unsigned char *row, float *h) {
    const uint4 w0 = *reinterpret_cast<const uint4 *>(row), w1 = *reinterpret_cast<const uint4 *>(row + 16);
    float f[16];
    unpack8(w0, f);
    unpack8(w1, f + 8);
#pragma unroll
    for (uint32_t e = 0; e < 16; ++e) h[e] += f[e];
}

// named barrier 1 over the CT compute threads; returns the AND of `pred`
template <uint32_t CT>
__device__ __forceinline__ bool compute_all(bool pred) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.and.pred q, 1, %2, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)pred), "n"(CT)
        : "memory");
    return r != 0;
}

template <uint32_t CT>
__device__ __forceinline__ void compute_sync() {
    asm volatile("bar.sync 1, %0;" ::"n"(CT) : "memory");
}

template <uint32_t Q, uint32_t NU>
__global__ void __launch_bounds__(MtShape<Q, NU>::THREADS, 1)
    k_made_tc(const MtPlan p, uint32_t *seq, uint32_t buflen, uint32_t nseq, float *logq, uint64_t seed,
              int given, int32_t *status) {
    using S = MtShape<Q, NU>;
    constexpr uint32_t SL = S::SL, CT = S::CT, ST = S::ST, WST = S::WST, HG = S::HG;
    extern __shared__ unsigned char smem_raw[];
    const uint32_t base_addr = smem_addr(smem_raw);
    unsigned char *sm = smem_raw + ((1024u - (base_addr & 1023u)) & 1023u);
    unsigned char *A1 = sm;
    unsigned char *A2 = A1 + MT_A1_BYTES;
    unsigned char *ring = A2 + MT_A2_BYTES;
    unsigned char *wring = ring + ST * MT_STAGE_BYTES;
    float *red_lg = reinterpret_cast<float *>(wring + WST * MT_WSTAGE_BYTES);  // [2][Q][SL][128]
    float *red_h2 = red_lg + S::RED_LG / 4;                                    // [2][HG][SL][128]
    uint64_t *bars = reinterpret_cast<uint64_t *>(red_h2 + S::RED_H2 / 4);
    uint64_t *full = bars, *empty = bars + ST;
    uint64_t *wfull = bars + 2 * ST, *wempty = wfull + WST;
    uint64_t *bar_a1 = wempty + WST, *bar_a2 = bar_a1 + 1, *bar_mma = bar_a1 + 2, *bar_fin = bar_a1 + 3;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bar_a1 + 4);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    const uint32_t L = p.L, G = p.G, nb = p.nb;
    const uint32_t ntiles = (nseq + MT_M - 1) / MT_M;
    constexpr uint32_t W_MMA = CT / 32, W_PROD = W_MMA + 1, W_WPROD = W_MMA + 2;

    if (tid == 0) {
        for (uint32_t s = 0; s < ST; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (uint32_t s = 0; s < WST; ++s) {
            mbar_init(&wfull[s], 1);
            mbar_init(&wempty[s], CT);
        }
        mbar_init(bar_a1, CT);
        mbar_init(bar_a2, CT);
        mbar_init(bar_mma, 1);
        mbar_init(bar_fin, 1);
        *abort_flag = 0;
        fence_mbar_init();
    }
    if (warp == W_MMA) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                     "r"(MT_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == W_PROD) {
        // ------------------------------------------ MMA weight-tile producer
        if ((tid & 31) == 0)
            mt_produce<MtOp, ST, MT_STAGE_BYTES>(p.ops, p.nops, p.img, ring, full, empty, ntiles, abort_flag, status);
    } else if (warp == W_WPROD) {
        // ------------------------------------------ CUDA-core weight producer
        if ((tid & 31) == 0)
            mt_produce<MtWOp, WST, MT_WSTAGE_BYTES>(p.wops, p.nwops, p.wimg, wring, wfull, wempty, ntiles, abort_flag,
                                                    status);
    } else if (warp == W_MMA) {
        // ---------------------------------------------------- MMA issue
        if ((tid & 31) == 0) {
            uint32_t it = 0, na1 = 0, na2 = 0;
            bool ok = true;
            const uint32_t a1base = smem_addr(A1), a2base = smem_addr(A2), rbase = smem_addr(ring);
            for (uint32_t t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
                for (uint32_t b = 0; b < nb && ok; ++b) {
                    const uint32_t *bk = p.blk + b * MT_BLK;
                    if (!mbar_wait_bounded(bar_a1, na1++ & 1, abort_flag, WAIT_LIMIT_NS)) {
                        report(status, ST_TIMEOUT_FULL);
                        *abort_flag = 1;
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    for (uint32_t pass = 0; pass < 2 && ok; ++pass) {
                        if (pass == 1) {
                            // block 0 has no layer-2 product and every MMA of the
                            // previous tile completed before its last block began
                            if (b == 0)
                                mbar_arrive(bar_mma);
                            else
                                tc_commit(bar_mma);
                            if (!mbar_wait_bounded(bar_a2, na2++ & 1, abort_flag, WAIT_LIMIT_NS)) {
                                report(status, ST_TIMEOUT_FULL);
                                *abort_flag = 1;
                                ok = false;
                                break;
                            }
                            tc_fence_after();
                        }
                        const uint32_t lo = bk[4 + pass], hi = bk[5 + pass];
                        for (uint32_t o = lo; o < hi; ++o) {
                            const uint32_t s = it % ST;
                            if (!mbar_wait_bounded(&full[s], (it / ST) & 1, abort_flag, WAIT_LIMIT_NS)) {
                                report(status, ST_TIMEOUT_FULL);
                                *abort_flag = 1;
                                ok = false;
                                break;
                            }
                            tc_fence_after();
                            const MtOp op = p.ops[o];
                            const uint32_t idesc = mt_idesc(op.rows);
                            const uint32_t bb = rbase + s * MT_STAGE_BYTES;
                            const uint32_t ab = op.kind == 0 ? a1base + op.kc * (MT_M * 128) : a2base;
                            for (uint32_t kk = 0; kk < op.ksteps; ++kk)
                                mt_mma(tmem + op.dcol, umma_desc_sw128(ab + kk * 32), umma_desc_sw128(bb + kk * 32),
                                       idesc, (op.kind == 0 && op.first && kk == 0) ? 0u : 1u);
                            tc_commit(&empty[s]);
                            ++it;
                        }
                    }
                }
            }
            // every MMA issued has completed before the accumulators are freed
            tc_commit(bar_fin);
            mbar_wait_bounded(bar_fin, 0, nullptr, WAIT_LIMIT_NS);
        }
    } else {
        // ---------------------------------------------------- walkers
        const uint32_t lane = tid & 31, qd = warp & 3, sl = warp >> 2;
        const uint32_t m = 32 * qd + lane;
        const uint32_t lane_base = (32 * qd) << 16;
        const uint32_t v0 = 16 * sl;  // this thread's first unit of a block
        uint32_t nmma = 0, wit = 0, ph_lg = 0, ph_h2 = 0;
        bool ok = true;
        // a bounded wait all compute threads decide together: named-barrier
        // steps follow, and tcgen05.ld/st need whole warps
        auto wait_cta = [&](uint64_t *bar, uint32_t parity) {
            const bool got = compute_all<CT>(mbar_wait_bounded(bar, parity, abort_flag, WAIT_LIMIT_NS));
            if (!got) {
                report(status, ST_TIMEOUT_FULL);
                *abort_flag = 1;
            }
            return got;
        };
        for (uint32_t t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
            const uint32_t n = t * MT_M + m;
            const bool valid = n < nseq;
            float lq = 0.0f;
            uint32_t cw = 0;  // residues of the current sequence word
            for (uint32_t b = 0; b < nb && ok; ++b) {
                const uint32_t *bk = p.blk + b * MT_BLK;
                const uint32_t c1 = bk[0], n1 = bk[1], d2ok = bk[7], nch = bk[9];
                const uint32_t s0 = b * G, s1 = min(L, s0 + G);
                if (b == 0 && sl == 0) {
                    // the logits accumulator of this tile starts at zero
                    for (uint32_t c = 0; c < nb * p.N3; c += 16) tmem_zero16(tmem + lane_base + c);
                    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
                }
                tc_fence_before();
                mbar_arrive(bar_a1);

                // this slice's hidden-1 units: bias + inputs from sites < s0,
                // FP32 weight rows streamed 64 / q sites at a time
                float h1[16];
#pragma unroll
                for (uint32_t k = 0; k < 16; ++k) h1[k] = __ldg(&p.b1b[b * MT_NU + v0 + k]);
                constexpr uint32_t CS = MT_CROWS / Q;  // sites per layer-1 chunk
                asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");  // the words stored so far
                for (uint32_t c = 0; c < nch; ++c) {
                    const uint32_t s = wit % WST;
                    if (!wait_cta(&wfull[s], (wit / WST) & 1)) {
                        ok = false;
                        break;
                    }
                    ++wit;
                    const float *chunk = reinterpret_cast<const float *>(wring + s * MT_WSTAGE_BYTES);
                    const uint32_t jend = min(s0, CS * (c + 1));
                    // four sites (one sequence word) per step, their 16 loads together
                    for (uint32_t j = CS * c; j < jend; j += 4) {
                        const uint32_t word = tmem_ld1(tmem + lane_base + p.wcol + (j >> 2));
                        float4 w[4][4];
#pragma unroll
                        for (uint32_t jj = 0; jj < 4; ++jj) {
                            const uint32_t x = min((word >> (8 * jj)) & 0xffu, Q - 1);
                            const uint32_t rr = (j + jj - CS * c) * Q + x;
                            const float *row = chunk + rr * MT_NU;
                            const uint32_t sw = mt_rsw(rr);
#pragma unroll
                            for (uint32_t gg = 0; gg < 4; ++gg)
                                w[jj][gg] = *reinterpret_cast<const float4 *>(row + 4 * ((v0 / 4 + gg) ^ sw));
                        }
#pragma unroll
                        for (uint32_t jj = 0; jj < 4; ++jj)
#pragma unroll
                            for (uint32_t gg = 0; gg < 4; ++gg) {
                                h1[4 * gg] += w[jj][gg].x;
                                h1[4 * gg + 1] += w[jj][gg].y;
                                h1[4 * gg + 2] += w[jj][gg].z;
                                h1[4 * gg + 3] += w[jj][gg].w;
                            }
                    }
                    mbar_arrive(&wempty[s]);
                }
                if (!ok) break;
                // the block's in-block weights, held for its sites
                const uint32_t s23 = wit % WST;
                if (!wait_cta(&wfull[s23], (wit / WST) & 1)) {
                    ok = false;
                    break;
                }
                ++wit;
                const unsigned char *w2s = wring + s23 * MT_WSTAGE_BYTES;
                const unsigned char *w3s = w2s + MT_W2_BYTES;
                const unsigned char *w1s = w3s + MT_W3_BYTES;
                const float *par = reinterpret_cast<const float *>(w2s + MT_PAR_OFF);
                const int32_t *cnt = reinterpret_cast<const int32_t *>(par + MT_PAR_CNT);
                // layer-2 prefix of the block (and the logits accumulator)
                if (!wait_cta(bar_mma, nmma++ & 1)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                // this slice's layer-2 prefix values, once per block
                float d2r[16];
                {
                    uint32_t r16[16];
                    if (d2ok) tmem_ld16(tmem + lane_base + p.d2col + v0, r16);
#pragma unroll
                    for (uint32_t k = 0; k < 16; ++k) d2r[k] = (d2ok ? __uint_as_float(r16[k]) : 0.0f) + par[MT_PAR_B2 + v0 + k];
                }
                // the block's sequence words when they are given
                uint32_t gw[2] = {0u, 0u};
                if (given && valid) {
                    gw[0] = seq[(size_t)(s0 >> 2) * buflen + n];
                    if (s1 > s0 + 4) gw[1] = seq[(size_t)((s0 >> 2) + 1) * buflen + n];
                }
                *reinterpret_cast<uint4 *>(A2 + m * 128 + ((((2 * sl) ^ (m & 7)) & 7) << 4)) = make_uint4(0, 0, 0, 0);
                *reinterpret_cast<uint4 *>(A2 + m * 128 + ((((2 * sl + 1) ^ (m & 7)) & 7) << 4)) =
                    make_uint4(0, 0, 0, 0);

                for (uint32_t i = s0; i < s1; ++i) {
                    const uint32_t il = i - s0;
                    // this slice's share of the logits of site i
                    {
                        float act2[16];
                        unpack8(*reinterpret_cast<const uint4 *>(A2 + m * 128 + ((((2 * sl) ^ (m & 7)) & 7) << 4)),
                                act2);
                        unpack8(*reinterpret_cast<const uint4 *>(A2 + m * 128 + ((((2 * sl + 1) ^ (m & 7)) & 7) << 4)),
                                act2 + 8);
                        float *rl = red_lg + (ph_lg & 1) * (Q * CT);
#pragma unroll
                        for (uint32_t a = 0; a < Q; ++a)
                            rl[(a * SL + sl) * MT_M + m] = dot16(w3s + (il * Q + a) * MT_ROW_BYTES + 2 * v0, act2);
                    }
                    float lg[Q];
                    if (b >= 1) {
                        tmem_ldq<Q>(tmem + lane_base + b * p.N3 + il * Q, lg);
                    } else {
#pragma unroll
                        for (uint32_t a = 0; a < Q; ++a) lg[a] = 0.0f;
                    }
                    compute_sync<CT>();
                    {
                        const float *rl = red_lg + (ph_lg & 1) * (Q * CT);
#pragma unroll
                        for (uint32_t a = 0; a < Q; ++a) {
                            float s = rl[(a * SL) * MT_M + m];
#pragma unroll
                            for (uint32_t k = 1; k < SL; ++k) s += rl[(a * SL + k) * MT_M + m];
                            lg[a] += par[MT_PAR_B3 + il * Q + a] + s;
                        }
                    }
                    ++ph_lg;
                    // draw (or read) residue i: the same in every slice
                    float mx = lg[0];
#pragma unroll
                    for (uint32_t a = 1; a < Q; ++a) mx = fmaxf(mx, lg[a]);
                    float ex[Q], se = 0.0f;
#pragma unroll
                    for (uint32_t a = 0; a < Q; ++a) {
                        ex[a] = expf(lg[a] - mx);
                        se += ex[a];
                    }
                    const float lse = mx + logf(se);
                    uint32_t r;
                    if (given) {
                        const uint32_t gword = il < 4 ? gw[0] : gw[1];
                        if ((i & 3) == 0) tmem_st1(tmem + lane_base + p.wcol + (i >> 2), gword);
                        r = min((gword >> (8 * (i & 3))) & 0xffu, Q - 1);
                    } else {
                        const float u = hash_uniform(seed, n, i) * se;
                        float c = 0.0f;
                        r = Q - 1;
                        bool found = false;
#pragma unroll
                        for (uint32_t a = 0; a < Q; ++a) {
                            c += ex[a];
                            if (!found && u < c) {
                                r = a;
                                found = true;
                            }
                        }
                    }
                    float lr = lg[0];
#pragma unroll
                    for (uint32_t a = 1; a < Q; ++a) lr = (r == a) ? lg[a] : lr;
                    lq += lr - lse;
                    if (!given) {
                        cw |= r << (8 * (i & 3));
                        if ((i & 3) == 3 || i == L - 1) {
                            if (valid && sl == 0) seq[(size_t)(i >> 2) * buflen + n] = cw;
                            // every slice writes the same word: each reads back its own
                            tmem_st1(tmem + lane_base + p.wcol + (i >> 2), cw);
                            cw = 0;
                        }
                    }
                    // its input to this slice's hidden-1 units
                    add16h(w1s + (il * Q + r) * MT_ROW_BYTES + 2 * v0, h1);
                    // hidden-2 units of degree i + 1, HG per barrier
                    if (i + 1 < L) {
                        const int32_t ulo = cnt[il], uhi = cnt[il + 1];
                        if (ulo < uhi) {
                            float act1[16];
#pragma unroll
                            for (uint32_t k = 0; k < 16; ++k) act1[k] = bf16r(fmaxf(h1[k], 0.0f));
                            for (int32_t u0 = ulo; u0 < uhi; u0 += HG) {
                                float *rh = red_h2 + (ph_h2 & 1) * (HG * CT);
#pragma unroll
                                for (uint32_t k = 0; k < HG; ++k) {
                                    const uint32_t uk = (uint32_t)min(u0 + (int32_t)k, uhi - 1);
                                    rh[(k * SL + sl) * MT_M + m] = dot16(w2s + uk * MT_ROW_BYTES + 2 * v0, act1);
                                }
                                compute_sync<CT>();
#pragma unroll
                                for (uint32_t k = 0; k < HG; ++k) {
                                    const int32_t u = u0 + (int32_t)k;
                                    // the slice that owns unit u finishes it
                                    if (u < uhi && (uint32_t)u / 16 == sl) {
                                        const uint32_t ul = (uint32_t)u - v0;
                                        float d2 = d2r[0];
#pragma unroll
                                        for (uint32_t e = 1; e < 16; ++e) d2 = (ul == e) ? d2r[e] : d2;
                                        float s = rh[(k * SL) * MT_M + m];
#pragma unroll
                                        for (uint32_t e = 1; e < SL; ++e) s += rh[(k * SL + e) * MT_M + m];
                                        const float z = d2 + s;
                                        *reinterpret_cast<unsigned short *>(A2 + mt_sw(m, (uint32_t)u)) =
                                            __bfloat16_as_ushort(__float2bfloat16_rn(fmaxf(z, 0.0f)));
                                    }
                                }
                                ++ph_h2;
                            }
                        }
                    }
                }
                mbar_arrive(&wempty[s23]);
                // this slice's hidden-1 units are final: into A1 for later blocks
                if (v0 < n1) {
#pragma unroll
                    for (uint32_t g = 0; g < 2; ++g) {
                        const uint32_t k = c1 + v0 + 8 * g;
                        uint4 w;
                        w.x = pack_bf16x2(fmaxf(h1[8 * g], 0.0f), fmaxf(h1[8 * g + 1], 0.0f));
                        w.y = pack_bf16x2(fmaxf(h1[8 * g + 2], 0.0f), fmaxf(h1[8 * g + 3], 0.0f));
                        w.z = pack_bf16x2(fmaxf(h1[8 * g + 4], 0.0f), fmaxf(h1[8 * g + 5], 0.0f));
                        w.w = pack_bf16x2(fmaxf(h1[8 * g + 6], 0.0f), fmaxf(h1[8 * g + 7], 0.0f));
                        *reinterpret_cast<uint4 *>(A1 + (k >> 6) * (MT_M * 128) + mt_sw(m, k & 63)) = w;
                    }
                }
                fence_proxy_async_smem();
                tc_fence_before();
                mbar_arrive(bar_a2);
            }
            if (ok && valid && sl == 0) logq[n] = lq;
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == W_MMA) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(MT_TMEM_COLS));
    }
}

// MMA weight tiles from the (bf16-valued) float weights.
__global__ void k_made_tc_images(const MtPlan p, unsigned char *img, const float *__restrict__ W2,
                                 const float *__restrict__ W3) {
    const MtOp op = p.ops[blockIdx.x];
    const uint32_t *bk = p.blk + op.blk * MT_BLK;
    const uint32_t c1 = bk[0], c2 = bk[2], n2 = bk[3];
    const uint32_t H = p.H, q = p.q, G = p.G, N3 = p.N3, L = p.L;
    for (uint32_t e = threadIdx.x; e < op.rows * 64; e += blockDim.x) {
        const uint32_t r = e / 64, k = e % 64;
        float v = 0.0f;
        if (op.kind == 0) {
            const uint32_t u = c2 + r, hv = op.kc * 64 + k;
            if (hv < c1) v = W2[(size_t)u * H + hv];
        } else {
            const uint32_t col = op.dcol + r;  // logits column of a later block
            const uint32_t beta = col / N3, c = col % N3;
            const uint32_t i = beta * G + c / q, a = c % q;
            if (c < G * q && i < L && k < n2) v = W3[(size_t)(i * q + a) * H + c2 + k];
        }
        *reinterpret_cast<unsigned short *>(img + op.off + mt_sw(r, k)) =
            __bfloat16_as_ushort(__float2bfloat16_rn(v));
    }
}

// CUDA-core weight stages: layer-1 chunks [64 rows (j, a)][48 units] in
// FP32, and per block W2 [48][48], W3 [G q][48] and the layer-1 rows of the
// block's own sites [G q][48] in bf16.
__global__ void k_made_tc_wimages(const MtPlan p, unsigned char *wimg, const float *__restrict__ W1T,
                                  const float *__restrict__ W2, const float *__restrict__ W3,
                                  const float *__restrict__ b2, const float *__restrict__ b3) {
    const MtWOp op = p.wops[blockIdx.x];
    const uint32_t *bk = p.blk + op.blk * MT_BLK;
    const uint32_t c1 = bk[0], n1 = bk[1], c2 = bk[2], n2 = bk[3];
    const uint32_t H = p.H, q = p.q, G = p.G, L = p.L;
    if (op.kind == 0) {
        float *out = reinterpret_cast<float *>(wimg + op.off);
        for (uint32_t e = threadIdx.x; e < MT_CROWS * MT_NU; e += blockDim.x) {
            const uint32_t r = e / MT_NU, x = e % MT_NU;
            const uint32_t j = (MT_CROWS / q) * op.chunk + r / q, a = r % q;
            out[r * MT_NU + 4 * ((x / 4) ^ mt_rsw(r)) + x % 4] =
                (j < L && x < n1) ? W1T[(size_t)(j * q + a) * H + c1 + x] : 0.0f;
        }
        return;
    }
    unsigned short *out = reinterpret_cast<unsigned short *>(wimg + op.off);
    const uint32_t s0 = op.blk * G;
    float *par = reinterpret_cast<float *>(wimg + op.off + MT_PAR_OFF);
    for (uint32_t e = threadIdx.x; e < MT_PAR_CNT + 16; e += blockDim.x) {
        if (e < MT_PAR_B2) {  // b3 of the block's sites
            const uint32_t i = s0 + e / q;
            par[e] = (e < G * q && i < L) ? b3[s0 * q + e] : 0.0f;
        } else if (e < MT_PAR_CNT) {
            const uint32_t u = e - MT_PAR_B2;
            par[e] = u < n2 ? b2[c2 + u] : 0.0f;
        } else {
            const uint32_t d = min(L, s0 + 1 + (e - MT_PAR_CNT));
            reinterpret_cast<int32_t *>(par)[e] = p.deg2_start[d] - (int32_t)c2;
        }
    }
    for (uint32_t e = threadIdx.x; e < MT_PAR_OFF / 2; e += blockDim.x) {
        const uint32_t r = e / MT_NU, x = e % MT_NU;
        float v = 0.0f;
        if (r < MT_NU) {
            if (r < n2 && x < n1) v = W2[(size_t)(c2 + r) * H + c1 + x];
        } else if (r < MT_NU + MT_GQMAX) {
            const uint32_t c = r - MT_NU, i = s0 + c / q;
            if (c < G * q && i < L && x < n2) v = W3[(size_t)(s0 * q + c) * H + c2 + x];
        } else {
            const uint32_t c = r - MT_NU - MT_GQMAX, i = s0 + c / q;
            if (c < G * q && i < L && x < n1) v = W1T[(size_t)(s0 * q + c) * H + c1 + x];
        }
        out[e] = __bfloat16_as_ushort(__float2bfloat16_rn(v));
    }
}

__global__ void k_made_tc_bias(const MtPlan p, float *b1b, float *b2b, float *b3c, const float *__restrict__ b1,
                               const float *__restrict__ b2, const float *__restrict__ b3) {
    const uint32_t nbias = p.nb * MT_NU, Lq = p.L * p.q;
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < 2 * nbias + Lq; e += gridDim.x * blockDim.x) {
        if (e < 2 * nbias) {
            const uint32_t x = e % nbias, b = x / MT_NU, v = x % MT_NU;
            const uint32_t *bk = p.blk + b * MT_BLK;
            if (e < nbias)
                b1b[x] = v < bk[1] ? b1[bk[0] + v] : 0.0f;
            else
                b2b[x] = v < bk[3] ? b2[bk[2] + v] : 0.0f;
        } else {
            b3c[e - 2 * nbias] = b3[e - 2 * nbias];
        }
    }
}

struct MtLayout {
    size_t ops, wops, blk, deg, img, wimg, b1b, b2b, b3, total;
};

static size_t mt_align(size_t x) { return (x + 255) & ~(size_t)255; }

static MtLayout mt_layout(uint32_t L, uint32_t q, uint32_t nb, size_t nops, size_t nwops, size_t img_bytes,
                          size_t wimg_bytes) {
    MtLayout o;
    size_t at = 0;
    auto take = [&](size_t bytes) {
        const size_t here = at;
        at = mt_align(at + bytes);
        return here;
    };
    o.ops = take(nops * sizeof(MtOp));
    o.wops = take(nwops * sizeof(MtWOp));
    o.blk = take((size_t)nb * MT_BLK * 4);
    o.deg = take((size_t)(L + 1) * 4);
    o.img = take(img_bytes);
    o.wimg = take(wimg_bytes);
    o.b1b = take((size_t)nb * MT_NU * 4);
    o.b2b = take((size_t)nb * MT_NU * 4);
    o.b3 = take((size_t)L * q * 4);
    o.total = at;
    return o;
}

// The host-side plan: block table, op lists and image sizes, or an error text.
struct MtHostPlan {
    uint32_t nb = 0, N3 = 0, d2col = 0, wcol = 0, nu = 16;
    std::vector<uint32_t> blk;
    std::vector<MtOp> ops;
    std::vector<MtWOp> wops;
    std::vector<int32_t> deg2;
    size_t img_bytes = 0, wimg_bytes = 0;
    const char *err = nullptr;
};

static MtHostPlan mt_plan(uint32_t L, uint32_t q, uint32_t H, uint32_t G, const int32_t *m1, const int32_t *m2) {
    MtHostPlan h;
    if (L < 2 || (q != 4 && q != 8) || H == 0 || H > MT_HMAX || H % 16 || (G != 4 && G != 8) ||
        G * q > MT_GQMAX) {
        h.err = "mi3_made_tc: needs q in {4, 8}, H <= 512 a multiple of 16, G in {4, 8} with G q <= 32";
        return h;
    }
    h.nb = (L + G - 1) / G;
    h.N3 = (G * q + 15) / 16 * 16;
    h.d2col = h.nb * h.N3;
    h.wcol = h.d2col + MT_NU;
    if (h.wcol + (L + 3) / 4 > MT_TMEM_COLS) {
        h.err = "mi3_made_tc: tensor memory too small (nb * roundup(G q, 16) + 48 + ceil(L/4) > 512)";
        return h;
    }
    std::vector<uint32_t> n1(h.nb, 0), n2(h.nb, 0);
    for (uint32_t k = 0; k < H; ++k) {
        if (m1[k] < 1 || m1[k] > (int32_t)L - 1 || m2[k] < 1 || m2[k] > (int32_t)L - 1 ||
            (k > 0 && (m1[k] < m1[k - 1] || m2[k] < m2[k - 1]))) {
            h.err = "mi3_made_tc: hidden degrees must be sorted and in [1, L-1]";
            return h;
        }
        ++n1[(m1[k] - 1) / G];
        ++n2[(m2[k] - 1) / G];
    }
    h.blk.assign((size_t)h.nb * MT_BLK, 0);
    uint32_t c1 = 0, c2 = 0, off = 0, woff = 0;
    for (uint32_t b = 0; b < h.nb; ++b) {
        if (n1[b] % 16 || n2[b] % 16 || n1[b] > MT_NU || n2[b] > MT_NU) {
            h.err = "mi3_made_tc: each degree block needs 0, 16, 32 or 48 units per layer";
            return h;
        }
        h.nu = std::max(h.nu, std::max(n1[b], n2[b]));
        uint32_t *bk = &h.blk[(size_t)b * MT_BLK];
        bk[0] = c1;
        bk[1] = n1[b];
        bk[2] = c2;
        bk[3] = n2[b];
        bk[4] = (uint32_t)h.ops.size();
        if (b >= 1 && n2[b] > 0 && c1 > 0) {
            for (uint32_t kc = 0; kc * 64 < c1; ++kc) {
                MtOp op{off, n2[b], kc, std::min<uint32_t>(64, c1 - 64 * kc) / 16, h.d2col, kc == 0 ? 1u : 0u, 0, b};
                h.ops.push_back(op);
                off += n2[b] * 128;
            }
        }
        bk[5] = (uint32_t)h.ops.size();
        if (b + 1 < h.nb && n2[b] > 0) {
            const uint32_t R = (h.nb - 1 - b) * h.N3;
            for (uint32_t r0 = 0; r0 < R; r0 += MT_STAGE_ROWS) {
                const uint32_t rows = std::min<uint32_t>(MT_STAGE_ROWS, R - r0);
                MtOp op{off, rows, 0, n2[b] / 16, (b + 1) * h.N3 + r0, 0, 1, b};
                h.ops.push_back(op);
                off += rows * 128;
            }
        }
        bk[6] = (uint32_t)h.ops.size();
        bk[7] = bk[5] > bk[4] ? 1u : 0u;
        // the CUDA-core weights: layer-1 chunks of the sites < s0, then the
        // block's in-block weights
        const uint32_t cs = MT_CROWS / q;
        const uint32_t nch = (b * G + cs - 1) / cs;
        bk[8] = (uint32_t)h.wops.size();
        bk[9] = nch;
        for (uint32_t c = 0; c < nch; ++c) {
            MtWOp w{woff, MT_CROWS * MT_NU * 4, 0, b, c, 0, 0, 0};
            h.wops.push_back(w);
            woff += w.bytes;
        }
        MtWOp w{woff, MT_W123_BYTES, 1, b, 0, 0, 0, 0};
        h.wops.push_back(w);
        woff += w.bytes;
        c1 += n1[b];
        c2 += n2[b];
    }
    h.img_bytes = off;
    h.wimg_bytes = woff;
    h.deg2.assign(L + 1, (int32_t)H);
    for (uint32_t d = 0; d <= L; ++d) {
        uint32_t k = 0;
        while (k < H && m2[k] < (int32_t)d) ++k;
        h.deg2[d] = (int32_t)k;
    }
    return h;
}

}  // namespace mi3

using namespace mi3;

extern "C" uint64_t mi3_made_tc_workspace(uint32_t L, uint32_t q, uint32_t H, uint32_t G, const int32_t *m1,
                                          const int32_t *m2) {
    if (!m1 || !m2) return 0;
    MtHostPlan h = mt_plan(L, q, H, G, m1, m2);
    if (h.err) return 0;
    return mt_layout(L, q, h.nb, h.ops.size(), h.wops.size(), h.img_bytes, h.wimg_bytes).total;
}

extern "C" int mi3_made_tc_prepare(uint32_t L, uint32_t q, uint32_t H, uint32_t G, const int32_t *m1,
                                   const int32_t *m2, const float *W1T, const float *b1, const float *W2,
                                   const float *b2, const float *W3, const float *b3, void *workspace,
                                   uint64_t ws_bytes, uint64_t *plan_out, void *stream) {
    if (!m1 || !m2 || !W1T || !b1 || !W2 || !b2 || !W3 || !b3 || !workspace || !plan_out)
        return fail(MI3_ERR_ARG, "mi3_made_tc_prepare: null pointer");
    MtHostPlan h = mt_plan(L, q, H, G, m1, m2);
    if (h.err) return fail(MI3_ERR_ARG, h.err);
    const MtLayout lay = mt_layout(L, q, h.nb, h.ops.size(), h.wops.size(), h.img_bytes, h.wimg_bytes);
    if (ws_bytes < lay.total) return fail(MI3_ERR_WORKSPACE, "mi3_made_tc_prepare: workspace too small");
    if (!aligned(workspace, 256)) return fail(MI3_ERR_ALIGN, "mi3_made_tc_prepare: workspace alignment");
    cudaStream_t st = as_stream(stream);
    unsigned char *ws = reinterpret_cast<unsigned char *>(workspace);
    if ((!h.ops.empty() &&
         cudaMemcpyAsync(ws + lay.ops, h.ops.data(), h.ops.size() * sizeof(MtOp), cudaMemcpyHostToDevice, st) !=
             cudaSuccess) ||
        cudaMemcpyAsync(ws + lay.wops, h.wops.data(), h.wops.size() * sizeof(MtWOp), cudaMemcpyHostToDevice, st) !=
            cudaSuccess ||
        cudaMemcpyAsync(ws + lay.blk, h.blk.data(), h.blk.size() * 4, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(ws + lay.deg, h.deg2.data(), h.deg2.size() * 4, cudaMemcpyHostToDevice, st) != cudaSuccess)
        return check_launch("mi3_made_tc_prepare: tables");
    MtPlan p;
    std::memset(&p, 0, sizeof(p));
    p.L = L;
    p.q = q;
    p.H = H;
    p.G = G;
    p.nb = h.nb;
    p.N3 = h.N3;
    p.d2col = h.d2col;
    p.wcol = h.wcol;
    p.nu = h.nu;
    p.nops = (uint32_t)h.ops.size();
    p.nwops = (uint32_t)h.wops.size();
    p.img_bytes = h.img_bytes;
    p.wimg_bytes = h.wimg_bytes;
    p.ops = reinterpret_cast<const MtOp *>(ws + lay.ops);
    p.wops = reinterpret_cast<const MtWOp *>(ws + lay.wops);
    p.blk = reinterpret_cast<const uint32_t *>(ws + lay.blk);
    p.deg2_start = reinterpret_cast<const int32_t *>(ws + lay.deg);
    p.img = ws + lay.img;
    p.wimg = ws + lay.wimg;
    p.b1b = reinterpret_cast<const float *>(ws + lay.b1b);
    p.b2b = reinterpret_cast<const float *>(ws + lay.b2b);
    p.b3 = reinterpret_cast<const float *>(ws + lay.b3);
    int rc;
    if (p.nops > 0) {
        k_made_tc_images<<<p.nops, 256, 0, st>>>(p, ws + lay.img, W2, W3);
        if ((rc = check_launch("mi3_made_tc_prepare: images"))) return rc;
    }
    k_made_tc_wimages<<<p.nwops, 256, 0, st>>>(p, ws + lay.wimg, W1T, W2, W3, b2, b3);
    if ((rc = check_launch("mi3_made_tc_prepare: weight stages"))) return rc;
    k_made_tc_bias<<<32, 256, 0, st>>>(p, reinterpret_cast<float *>(ws + lay.b1b),
                                       reinterpret_cast<float *>(ws + lay.b2b), reinterpret_cast<float *>(ws + lay.b3),
                                       b1, b2, b3);
    if ((rc = check_launch("mi3_made_tc_prepare: biases"))) return rc;
    std::memset(plan_out, 0, 24 * 8);
    std::memcpy(plan_out, &p, sizeof(p));
    return MI3_OK;
}

extern "C" int mi3_made_tc_sample(const uint64_t *plan, uint32_t *seq, uint32_t buflen, uint32_t nseq, float *logq,
                                  uint64_t seed, int32_t given, int32_t *status, void *stream) {
    if (!plan || !seq || !logq || !status) return fail(MI3_ERR_ARG, "mi3_made_tc_sample: null pointer");
    MtPlan p;
    std::memcpy(&p, plan, sizeof(p));
    if (!p.wops || !p.blk || p.nb == 0 || (p.q != 4 && p.q != 8))
        return fail(MI3_ERR_ARG, "mi3_made_tc_sample: plan not prepared");
    if (nseq > buflen) return fail(MI3_ERR_ARG, "mi3_made_tc_sample: nseq > buflen");
    if (nseq == 0) return MI3_OK;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const uint32_t ntiles = (nseq + MT_M - 1) / MT_M;
    const uint32_t grid = std::min<uint32_t>(ntiles, (uint32_t)nsm);
    cudaStream_t st = as_stream(stream);
    // 1, 2 or 3 unit slices per walker for 16, 32 or 48 units per block and layer
    auto launch = [&](auto kern, uint32_t threads, uint32_t smem) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<grid, threads, smem, st>>>(p, seq, buflen, nseq, logq, seed, given, status);
    };
    if (p.q == 4) {
        if (p.nu <= 16)
            launch(k_made_tc<4, 16>, MtShape<4, 16>::THREADS, MtShape<4, 16>::SMEM);
        else if (p.nu <= 32)
            launch(k_made_tc<4, 32>, MtShape<4, 32>::THREADS, MtShape<4, 32>::SMEM);
        else
            launch(k_made_tc<4, 48>, MtShape<4, 48>::THREADS, MtShape<4, 48>::SMEM);
    } else {
        if (p.nu <= 16)
            launch(k_made_tc<8, 16>, MtShape<8, 16>::THREADS, MtShape<8, 16>::SMEM);
        else if (p.nu <= 32)
            launch(k_made_tc<8, 32>, MtShape<8, 32>::THREADS, MtShape<8, 32>::SMEM);
        else
            launch(k_made_tc<8, 48>, MtShape<8, 48>::THREADS, MtShape<8, 48>::SMEM);
    }
    return check_launch("mi3_made_tc_sample");
}
