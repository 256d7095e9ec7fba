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

#include <algorithm>
#include <utility>
#include <vector>

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

// ---------------------------------------------------------------------------
// Host side (shared by the host generator, the device builder's planning and
// the CPU oracle's copy of the generator).
// ---------------------------------------------------------------------------
struct GenProj {
    int32_t src_pop, dst_pop;
    uint64_t pseed;
};

// Remote projection choice of one generated network.
struct GenPlan {
    std::vector<GenProj> proj;              // creation order
    std::vector<std::vector<int>> in, out;  // per population: projection ids in creation order
};

inline GenPlan gen_plan(const bsim_gen_spec &g)
{
    GenPlan pl;
    const int P = g.n_pop;
    pl.in.assign(P, {});
    pl.out.assign(P, {});
    for (int k = 0; k + 1 < P; k++) pl.proj.push_back({k, k + 1, proj_seed(g.seed, k)});
    if (P >= 2) {
        int m = (int)(g.remote_frac * (float)P + 0.5f);
        m = std::min(m, P);
        std::vector<std::pair<uint64_t, int>> keys;
        for (int k = 0; k < P; k++) keys.push_back({hash3(g.seed ^ SALT_REMOTE_SEL, (uint64_t)k, 0), k});
        std::sort(keys.begin(), keys.end());
        std::vector<int> sel;
        for (int r = 0; r < m; r++) sel.push_back(keys[r].second);
        std::sort(sel.begin(), sel.end());
        for (int k : sel) {
            uint64_t h = hash3(g.seed ^ SALT_REMOTE_TGT, (uint64_t)k, 0);
            int tgt = (int)((k + 1 + (int64_t)(h % (uint64_t)(P - 1))) % P);
            int id = (int)pl.proj.size();
            pl.proj.push_back({k, tgt, proj_seed(g.seed, id)});
        }
    }
    for (int id = 0; id < (int)pl.proj.size(); id++) {
        pl.out[pl.proj[id].src_pop].push_back(id);
        pl.in[pl.proj[id].dst_pop].push_back(id);
    }
    return pl;
}

// LIFENeuron constructor arguments of one generated neuron.
inline void spec_params(const bsim_gen_spec &g, float ioff, float vinit, float *p)
{
    p[0] = vinit; p[1] = g.v_rest; p[2] = g.v_reset; p[3] = g.cm; p[4] = g.tau_m;
    p[5] = g.tau_refrac; p[6] = g.tau_syn_E; p[7] = g.tau_syn_I; p[8] = g.v_thresh; p[9] = ioff;
}

// The whole network as flat arrays in global creation order (any output may be
// NULL; with src NULL only the sizes are produced). The spec must be valid.
inline void netgen_host(const bsim_gen_spec &g, float *params, int32_t *pop, int32_t *src, int32_t *dst, float *w,
                        int32_t *d, int64_t *n_out, int64_t *s_out)
{
    GenPlan pl = gen_plan(g);
    const int64_t n = (int64_t)g.n_pop * g.pop_size;
    if (params || pop) {
        for (int64_t i = 0; i < n; i++) {
            float ioff, vinit;
            draw_neuron(g.seed, (uint64_t)i, g, &ioff, &vinit);
            if (params) spec_params(g, ioff, vinit, params + 10 * i);
            if (pop) pop[i] = (int32_t)(i / g.pop_size);
        }
    }
    const uint32_t p24 = prob24(g.p_conn), exc24 = prob24(g.exc_frac);
    const float w_exc = g.w_max, w_inh = g.inh_scale * g.w_max;
    int64_t s = 0;
    for (const GenProj &pr : pl.proj) {
        for (int64_t i = 0; i < g.pop_size; i++) {
            for (int64_t j = 0; j < g.pop_size; j++) {
                SynDraw sd;
                if (!draw_pair(pr.pseed, (uint64_t)i, (uint64_t)j, p24, exc24, w_exc, w_inh, g.max_delay, &sd)) continue;
                if (src) {
                    src[s] = (int32_t)(pr.src_pop * (int64_t)g.pop_size + i);
                    dst[s] = (int32_t)(pr.dst_pop * (int64_t)g.pop_size + j);
                    w[s] = sd.w;
                    d[s] = sd.d;
                }
                s++;
            }
        }
    }
    if (n_out) *n_out = n;
    if (s_out) *s_out = s;
}

}  // namespace bsim
