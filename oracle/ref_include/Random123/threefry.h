/*
 * Minimal Threefry-2x32 (20 rounds) for compiling the reference's CPU
 * generator, extras/mcmcCPUgenThreaded.c, which includes
 * "Random123/threefry.h" from the Random123 library (D. E. Shaw Research).
 * Random123 is not vendored in the reference and no version is pinned there.
 * This header restates the published Threefry-2x32 algorithm (Salmon, Moraes,
 * Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11; rotation
 * constants and key-schedule parity from the Threefish/Skein specification)
 * with the type and function names that the generator's call sites use
 * (mcmcCPUgenThreaded.c:89-104).  It serves only the timed CPU baseline; the
 * baseline's random stream is not part of any parity claim.
 */
#ifndef MI3_SHIM_THREEFRY_H
#define MI3_SHIM_THREEFRY_H
#include <stdint.h>

typedef struct { uint32_t v[2]; } threefry2x32_ctr_t;
typedef struct { uint32_t v[2]; } threefry2x32_key_t;

static inline uint32_t mi3_rotl32(uint32_t x, unsigned r) {
    return (x << r) | (x >> (32u - r));
}

static inline threefry2x32_ctr_t threefry2x32(threefry2x32_ctr_t in, threefry2x32_key_t k) {
    static const unsigned R[8] = {13, 15, 26, 6, 17, 29, 16, 24};
    uint32_t ks[3];
    ks[0] = k.v[0];
    ks[1] = k.v[1];
    ks[2] = 0x1BD11BDAu ^ k.v[0] ^ k.v[1];
    uint32_t x0 = in.v[0] + ks[0];
    uint32_t x1 = in.v[1] + ks[1];
    for (unsigned r = 0; r < 20; r++) {
        x0 += x1;
        x1 = mi3_rotl32(x1, R[r % 8]);
        x1 ^= x0;
        if ((r & 3u) == 3u) {
            unsigned s = (r + 1u) / 4u;
            x0 += ks[s % 3u];
            x1 += ks[(s + 1u) % 3u];
            x1 += s;
        }
    }
    threefry2x32_ctr_t out;
    out.v[0] = x0;
    out.v[1] = x1;
    return out;
}
#endif
