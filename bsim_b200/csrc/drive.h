// Input-drive neurons fed through the same step as LIF_brian: ConstantNeuron and
// PoissonNeuron (the reference's Constant_spikes / Poisson_spikes,
// include/Neuron.h:25-26), with the semantics of the reference's GPU kernels:
//
//   Constant  src/neuron/constant/constant.cu:18-22
//             fires at cycle t iff t < end_cycle and (t - start_cycle) * fire_rate > fire_count;
//             start/end cycles = (int)(time / dt) (ConstantNeuron.cpp:55-62)
//   Poisson   src/neuron/poisson/poisson.cu:29-31 and 9-15
//             fires at cycle t iff t == fire_cycle and t <= end_cycle, then
//             fire_cycle += 1 + Poisson(rate) + refrac_step; the first fire_cycle is
//             (int)(start_time / dt) + Poisson(rate) (PoissonNeuron.cpp:35-44).
//             `rate` is the mean of the Poisson-distributed gap, in cycles.
//
// The reference draws its Poisson numbers from a clock-seeded std::default_random_engine
// (first cycle) and curand (later gaps), so its spike trains are not reproducible. Here
// every draw is a pure function of (seed, instance-local neuron id, the cycle the draw
// is made for), identical on the host and the device:
//   Poisson(rate) = sum of Poisson(64 * 4^l) draws for the base-4 digits of
//   q = floor(rate / 64) (level l = 0..3 takes digit l, level 4 takes q >> 8), each by
//   inversion of a 32-bit uniform through a CDF table, plus Poisson(r), r = rate - 64 q,
//   by Knuth's product-of-uniforms method against exp(-r) (computed on the host).
// The tables are built on the host from the pmf recurrence p(k+1) = p(k) * mu / (k+1)
// in double precision (multiplications and divisions only), so any IEEE host builds
// the same thresholds.
#pragma once
#include <stdint.h>

#include <vector>

#include "netgen.h"

namespace bsim {

enum : uint64_t { SALT_POISSON = 0x706f6973736f6e5fULL };

constexpr int POISSON_LEVELS = 5;  // table means 64, 256, 1024, 4096, 16384

struct PoissonTables {
    const uint32_t *thr;               // all levels' thresholds, concatenated
    int32_t off[POISSON_LEVELS];       // first threshold of each level
    int32_t len[POISSON_LEVELS];       // thresholds per level (the last one is 0xffffffff)
    int32_t kmin[POISSON_LEVELS];      // value of a level's first threshold
};

// Largest rate the sampler takes (64 * q stays exact in fp32).
constexpr float POISSON_MAX_RATE = 16777216.0f;

// Key of the draw made for a neuron when it fires at cycle `cycle` (-1: the initial draw).
BSIM_HD uint64_t poisson_key(uint64_t seed, int64_t local_id, int64_t cycle)
{
    return hash3(seed ^ SALT_POISSON, (uint64_t)local_id, (uint64_t)(cycle + 1));
}

BSIM_HD uint64_t poisson_stream(uint64_t key, uint32_t i) { return mix64(key + (uint64_t)i * 0x9e3779b97f4a7c15ULL); }

// Smallest level index i with u < thr[i] (thr[len-1] = 0xffffffff, so i < len).
BSIM_HD int32_t poisson_invert(const uint32_t *thr, int32_t len, uint32_t u)
{
    int32_t lo = 0, hi = len - 1;
    while (lo < hi) {
        const int32_t mid = (lo + hi) >> 1;
        if (u < thr[mid]) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

// One Poisson(rate) draw. exp_neg_r = exp(-(rate - 64 * floor(rate / 64))), rounded to fp32.
BSIM_HD int32_t poisson_draw(uint64_t key, float rate, float exp_neg_r, const PoissonTables &T)
{
    const uint32_t q = (uint32_t)mul_rn_hd(rate, 0.015625f);  // floor(rate / 64), exact scaling
    uint32_t i = 0;
    int32_t k = 0;
    uint32_t rest = q;
    for (int l = 0; l < POISSON_LEVELS; l++) {
        const uint32_t cnt = l < POISSON_LEVELS - 1 ? (rest & 3u) : rest;
        rest >>= 2;
        for (uint32_t c = 0; c < cnt; c++) {
            const uint32_t u = (uint32_t)(poisson_stream(key, i++) >> 32);
            k += T.kmin[l] + poisson_invert(T.thr + T.off[l], T.len[l], u);
        }
    }
    float p = 1.0f;
    for (;;) {
        const uint32_t u24 = (uint32_t)(poisson_stream(key, i++) >> 40);
        p = mul_rn_hd(p, add_rn_hd((float)u24, 0.5f) * (1.0f / 16777216.0f));  // (0,1), exact
        if (p <= exp_neg_r) break;
        k++;
    }
    return k;
}

// Host: the thresholds of the five levels. Level l has mean mu = 64 * 4^l and
// standard deviation 8 * 2^l and covers mu +- 12 standard deviations (clipped at 0).
// Unnormalised pmf from the mode: w(mu) = 1, w(k+1) = w(k) * mu / (k+1) upwards,
// w(k-1) = w(k) * k / mu downwards; threshold i = floor(2^32 * sum_{k<=kmin+i} w / sum w),
// the last one 0xffffffff.
inline void poisson_build_tables(std::vector<uint32_t> &thr, int32_t off[POISSON_LEVELS],
                                 int32_t len[POISSON_LEVELS], int32_t kmin[POISSON_LEVELS])
{
    thr.clear();
    for (int l = 0; l < POISSON_LEVELS; l++) {
        const int64_t mu = 64LL << (2 * l), sd = 8LL << l;
        const int64_t lo = mu - 12 * sd < 0 ? 0 : mu - 12 * sd, hi = mu + 12 * sd;
        const int64_t m = hi - lo + 1;
        std::vector<double> w((size_t)m);
        w[(size_t)(mu - lo)] = 1.0;
        for (int64_t k = mu; k < hi; k++) w[(size_t)(k + 1 - lo)] = w[(size_t)(k - lo)] * (double)mu / (double)(k + 1);
        for (int64_t k = mu; k > lo; k--) w[(size_t)(k - 1 - lo)] = w[(size_t)(k - lo)] * (double)k / (double)mu;
        double total = 0.0;
        for (int64_t i = 0; i < m; i++) total += w[(size_t)i];
        off[l] = (int32_t)thr.size();
        len[l] = (int32_t)m;
        kmin[l] = (int32_t)lo;
        double c = 0.0;
        for (int64_t i = 0; i < m; i++) {
            c += w[(size_t)i];
            const double f = c / total * 4294967296.0;
            uint32_t t = f >= 4294967295.0 ? 0xffffffffu : (uint32_t)f;
            if (i == m - 1) t = 0xffffffffu;
            thr.push_back(t);
        }
    }
}

}  // namespace bsim
