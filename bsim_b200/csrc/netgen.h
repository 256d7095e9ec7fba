// Seeded synthetic network generator shared by the host builder and the device
// builder (the same integer and fp32 arithmetic on both sides, so the two give
// bit-identical networks).
//
// Workload shape (the reference's standard_test generator, test/gpu/standard_test.cpp:54-153,
// replaced by a sparse random variant): P populations of n LIF_brian neurons; a
// chain projection k -> k+1 (no wrap-around) for k = 0..P-2, then a seeded
// round(remote_frac * P) of the populations each add one projection to a
// uniformly chosen other population. Every projection connects each (src, dst)
// pair independently with probability p_conn. A synapse is excitatory with
// probability exc_frac, weight U[0, w_max), else inhibitory with weight
// -U[0, inh_scale * w_max); its delay is U{1..max_delay} steps. Every neuron
// draws i_offset from U[i_min, i_max) and v_init from U[v_init_lo, v_init_hi).
//
// Creation order (the order a program would call Network::connect): chain
// projections by source population, then remote projections by source
// population; inside a projection source-major, target-minor.
#pragma once
#include <stdint.h>

#include "../../include/bsim_b200.h"

#if defined(__CUDACC__)
#define BSIM_HD __host__ __device__ __forceinline__
#else
#define BSIM_HD inline
#endif

namespace bsim {

// Stafford's "Mix13" 64-bit finaliser (as used by SplitMix64).
BSIM_HD uint64_t mix64(uint64_t x)
{
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ULL;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebULL;
    x ^= x >> 31;
    return x;
}

BSIM_HD uint64_t hash3(uint64_t seed, uint64_t a, uint64_t b)
{
    return mix64(mix64(seed ^ (a * 0x9e3779b97f4a7c15ULL)) + b * 0xd1b54a32d192ed03ULL + 1);
}

enum : uint64_t {
    SALT_NEURON = 0x6e6575726f6e5f31ULL,
    SALT_REMOTE_SEL = 0x72656d6f74655f73ULL,
    SALT_REMOTE_TGT = 0x72656d6f74655f74ULL,
    SALT_PROJ = 0x70726f6a5f736565ULL,
    SALT_SYN = 0x73796e5f76616c73ULL,
};

// 24-bit thresholds for Bernoulli draws taken from the top 24 bits of a hash.
BSIM_HD uint32_t prob24(float p)
{
    if (!(p > 0.0f)) return 0u;
    if (p >= 1.0f) return 1u << 24;
    return (uint32_t)(p * 16777216.0f + 0.5f);
}

#if defined(__CUDACC__)
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
#define BSIM_RN_MUL(a, b) mul_rn_hd(a, b)
BSIM_HD float mul_rn_hd(float a, float b)
{
#if defined(__CUDA_ARCH__)
    return __fmul_rn(a, b);
#else
    volatile float r = a * b;
    return r;
#endif
}
BSIM_HD float add_rn_hd(float a, float b)
{
#if defined(__CUDA_ARCH__)
    return __fadd_rn(a, b);
#else
    volatile float r = a + b;
    return r;
#endif
}
#else
inline float mul_rn_hd(float a, float b) { volatile float r = a * b; return r; }
inline float add_rn_hd(float a, float b) { volatile float r = a + b; return r; }
#endif

// u in [0,1) with 24 significant bits: exact in fp32.
BSIM_HD float unit24(uint32_t u24) { return (float)u24 * (1.0f / 16777216.0f); }

// One synapse's value for a connected pair. Returns false when not connected.
struct SynDraw {
    float w;
    int32_t d;
};

BSIM_HD bool draw_pair(uint64_t proj_seed, uint64_t i, uint64_t j, uint32_t p24, uint32_t exc24,
                       float w_exc, float w_inh, int32_t max_delay, SynDraw *out)
{
    uint64_t h = hash3(proj_seed, i, j);
    if ((uint32_t)(h >> 40) >= p24) return false;
    uint64_t h2 = mix64(h ^ SALT_SYN);
    float u = unit24((uint32_t)(h2 >> 16) & 0xFFFFFFu);
    if ((uint32_t)(h2 >> 40) < exc24) {
        out->w = mul_rn_hd(u, w_exc);
    } else {
        out->w = -mul_rn_hd(u, w_inh);
    }
    out->d = 1 + (int32_t)(((h2 & 0xFFFFull) * (uint64_t)max_delay) >> 16);
    return true;
}

// Per-neuron drawn parameters.
BSIM_HD void draw_neuron(uint64_t seed, uint64_t gid_local, const bsim_gen_spec &g, float *i_offset, float *v_init)
{
    uint64_t h = hash3(seed ^ SALT_NEURON, gid_local, 0);
    float u1 = unit24((uint32_t)(h >> 40));
    float u2 = unit24((uint32_t)(h >> 16) & 0xFFFFFFu);
    *i_offset = add_rn_hd(g.i_min, mul_rn_hd(u1, g.i_max - g.i_min));
    *v_init = add_rn_hd(g.v_init_lo, mul_rn_hd(u2, g.v_init_hi - g.v_init_lo));
}

BSIM_HD uint64_t proj_seed(uint64_t seed, int32_t proj) { return hash3(seed ^ SALT_PROJ, (uint64_t)proj, 7); }

}  // namespace bsim
