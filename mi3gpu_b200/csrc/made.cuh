// made.cuh -- pieces shared by the MADE proposal kernels (made.cu, made_tc.cu).
#pragma once
#include "common.cuh"

namespace mi3 {

// Counter-based uniform in [0,1): splitmix64 finaliser of (seed, n, i).
__device__ __forceinline__ float hash_uniform(uint64_t seed, uint64_t n, uint64_t i) {
    uint64_t z = seed + 0x9E3779B97F4A7C15ull * (n * 0x100000001B3ull + i + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (float)(z >> 40) * 0x1.0p-24f;
}

}  // namespace mi3
