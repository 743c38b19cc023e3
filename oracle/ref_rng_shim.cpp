// ref_rng_shim.cpp -- compiles the reference's own MWC64X OpenCL source
// (mi3gpu/mwc64x/cl/mwc64x/{skip_mwc,mwc64x_rng,mwc64xvec2_rng}.cl) as C++ so
// that the oracle's restatement of the generator can be pinned against it.
//
// TEST INFRASTRUCTURE ONLY: built into oracle/_ref by oracle/Makefile, loaded
// by the tests.  Nothing here is part of the library.
//
// The shim supplies the OpenCL C vocabulary those files use: `uint` as a
// 32-bit class type (so that the OpenCL vector literal `(uint2)(a, b)` can be
// formed through an overloaded comma), `uint2`/`int2` with the element-wise
// operators the generator needs, `mad_hi`, `as_uint2` and `get_global_id`.
#include <cstdint>
#include <cstddef>

namespace clshim {

struct U32;
struct U32pair;

struct U32 {
    uint32_t v;
    U32() : v(0) {}
    U32(unsigned long long x) : v((uint32_t)x) {}
    U32(unsigned long x) : v((uint32_t)x) {}
    U32(unsigned int x) : v(x) {}
    U32(int x) : v((uint32_t)x) {}
    U32(bool x) : v(x ? 1u : 0u) {}
    operator uint32_t() const { return v; }
};

struct U32pair { U32 a, b; };
inline U32pair operator,(U32 a, U32 b) { return U32pair{a, b}; }

struct I2 { int32_t x, y; };

struct U2 {
    U32 x, y;
    U2() {}
    U2(uint32_t s) : x(s), y(s) {}
    U2(U32pair p) : x(p.a), y(p.b) {}
};

inline U2 mk(uint32_t a, uint32_t b) { U2 r; r.x = a; r.y = b; return r; }
inline U2 operator*(unsigned long long s, U2 v) {
    return mk((uint32_t)s * (uint32_t)v.x, (uint32_t)s * (uint32_t)v.y);
}
inline U2 operator+(U2 a, U2 b) { return mk((uint32_t)a.x + (uint32_t)b.x, (uint32_t)a.y + (uint32_t)b.y); }
inline U2 operator^(U2 a, U2 b) { return mk((uint32_t)a.x ^ (uint32_t)b.x, (uint32_t)a.y ^ (uint32_t)b.y); }
// OpenCL vector relational operators return -1 (all bits set) for true.
inline I2 operator<(U2 a, U2 b) {
    return I2{((uint32_t)a.x < (uint32_t)b.x) ? -1 : 0, ((uint32_t)a.y < (uint32_t)b.y) ? -1 : 0};
}
inline I2 operator-(I2 a) { return I2{-a.x, -a.y}; }
inline U2 as_uint2(I2 a) { return mk((uint32_t)a.x, (uint32_t)a.y); }

inline uint32_t mad_hi(uint32_t a, uint32_t b, uint32_t c) {
    return (uint32_t)(((uint64_t)a * (uint64_t)b) >> 32) + c;
}
inline U2 mad_hi(U2 a, U2 b, U2 c) {
    return mk(mad_hi((uint32_t)a.x, (uint32_t)b.x, (uint32_t)c.x),
              mad_hi((uint32_t)a.y, (uint32_t)b.y, (uint32_t)c.y));
}

static size_t g_global_id = 0;
inline size_t get_global_id(int) { return g_global_id; }

}  // namespace clshim

using namespace clshim;
#define uint U32
#define uint2 U2
#define ulong unsigned long
#define s0 x
#define s1 y

#include "mwc64x/cl/mwc64x/skip_mwc.cl"
#include "mwc64x/cl/mwc64x/mwc64x_rng.cl"
#include "mwc64x/cl/mwc64x/mwc64xvec2_rng.cl"

#undef uint
#undef uint2
#undef ulong
#undef s0
#undef s1

// ---- C entry points used by the tests -------------------------------------
// State image per walker: uint32[4] = {x.s0, x.s1, c.s0, c.s1}.
static void put(uint32_t *st, const mwc64xvec2_state_t &s) {
    st[0] = s.x.x; st[1] = s.x.y; st[2] = s.c.x; st[3] = s.c.y;
}
static mwc64xvec2_state_t get(const uint32_t *st) {
    mwc64xvec2_state_t s;
    s.x = mk(st[0], st[1]);
    s.c = mk(st[2], st[3]);
    return s;
}

extern "C" {

// initRNG2 (mcmc.cl:349-356) for work items 0..n-1.
void ref_init_rng2(uint32_t *states, uint32_t n, uint64_t offset, uint64_t span) {
    for (uint32_t g = 0; g < n; g++) {
        g_global_id = g;
        mwc64xvec2_state_t s;
        MWC64XVEC2_SeedStreams(&s, offset, span);
        put(&states[4*g], s);
    }
}

// `count` calls of MWC64XVEC2_NextUint2 on one state; outputs 2*count words.
void ref_vec2_stream(uint32_t *state, uint32_t count, uint32_t *out) {
    mwc64xvec2_state_t s = get(state);
    for (uint32_t i = 0; i < count; i++) {
        U2 r = MWC64XVEC2_NextUint2(&s);
        out[2*i] = r.x; out[2*i+1] = r.y;
    }
    put(state, s);
}

void ref_vec2_skip(uint32_t *state, uint64_t dist) {
    mwc64xvec2_state_t s = get(state);
    MWC64XVEC2_Skip(&s, dist);
    put(state, s);
}

// Scalar generator: seed stream gid with (base, gap); x,c out.
void ref_scalar_seed(uint64_t gid, uint64_t base, uint64_t gap, uint32_t *xc) {
    g_global_id = gid;
    mwc64x_state_t s;
    MWC64X_SeedStreams(&s, base, gap);
    xc[0] = s.x; xc[1] = s.c;
}

void ref_scalar_stream(uint32_t *xc, uint32_t count, uint32_t *out) {
    mwc64x_state_t s;
    s.x = xc[0]; s.c = xc[1];
    for (uint32_t i = 0; i < count; i++) out[i] = MWC64X_NextUint(&s);
    xc[0] = s.x; xc[1] = s.c;
}

void ref_scalar_skip(uint32_t *xc, uint64_t dist) {
    mwc64x_state_t s;
    s.x = xc[0]; s.c = xc[1];
    MWC64X_Skip(&s, dist);
    xc[0] = s.x; xc[1] = s.c;
}

}  // extern "C"
