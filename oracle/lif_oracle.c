/*
 * TEST INFRASTRUCTURE ONLY — the CPU oracle for the GPU engine (see
 * lif_oracle.h). Instantiates lif_oracle_impl.h for the reference's float
 * build and for its double build (-DUSE_DOUBLE, src/utils/constant.h:12-16).
 */
#include <math.h>
#include <stdlib.h>
#include <stdint.h>
#include <string.h>

#include "lif_oracle.h"

/* ---- the engine's Poisson sampler, restated (shared by both builds) ----
 * Poisson(rate) = sum of Poisson(64 * 4^l) draws for the base-4 digits of
 * q = floor(rate / 64) (digits 0..3 at levels 0..3, q >> 8 at level 4), each by
 * inversion of a 32-bit uniform through a CDF table, plus Poisson(rate - 64 q) by
 * Knuth's product of uniforms against exp(-(rate - 64 q)). Draws come from
 * SplitMix64's finaliser over (seed, neuron id, cycle, index). */
static uint64_t o_mix64(uint64_t x)
{
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ULL;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebULL;
    x ^= x >> 31;
    return x;
}

static uint64_t o_hash3(uint64_t seed, uint64_t a, uint64_t b)
{
    return o_mix64(o_mix64(seed ^ (a * 0x9e3779b97f4a7c15ULL)) + b * 0xd1b54a32d192ed03ULL + 1);
}

#define O_POISSON_SALT 0x706f6973736f6e5fULL
#define O_LEVELS 5

static uint32_t *o_thr = NULL;
static int32_t o_off[O_LEVELS], o_len[O_LEVELS], o_kmin[O_LEVELS];

/* CDF tables of Poisson(64 * 4^l) over mean +- 12 sd, from the pmf recurrence
 * around the mode in double precision. */
static int o_tables(void)
{
    if (o_thr) return 0;
    int64_t total_len = 0;
    for (int l = 0; l < O_LEVELS; l++) {
        int64_t mu = 64LL << (2 * l), sd = 8LL << l;
        int64_t lo = mu - 12 * sd < 0 ? 0 : mu - 12 * sd;
        total_len += mu + 12 * sd - lo + 1;
    }
    uint32_t *thr = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)total_len);
    if (!thr) return -4;
    int64_t at = 0;
    for (int l = 0; l < O_LEVELS; l++) {
        int64_t mu = 64LL << (2 * l), sd = 8LL << l;
        int64_t lo = mu - 12 * sd < 0 ? 0 : mu - 12 * sd, hi = mu + 12 * sd, m = hi - lo + 1;
        double *w = (double *)malloc(sizeof(double) * (size_t)m);
        if (!w) { free(thr); return -4; }
        w[mu - lo] = 1.0;
        for (int64_t k = mu; k < hi; k++) w[k + 1 - lo] = w[k - lo] * (double)mu / (double)(k + 1);
        for (int64_t k = mu; k > lo; k--) w[k - 1 - lo] = w[k - lo] * (double)k / (double)mu;
        double tot = 0.0, c = 0.0;
        for (int64_t i = 0; i < m; i++) tot += w[i];
        o_off[l] = (int32_t)at;
        o_len[l] = (int32_t)m;
        o_kmin[l] = (int32_t)lo;
        for (int64_t i = 0; i < m; i++) {
            c += w[i];
            double f = c / tot * 4294967296.0;
            uint32_t t = f >= 4294967295.0 ? 0xffffffffu : (uint32_t)f;
            thr[at++] = i == m - 1 ? 0xffffffffu : t;
        }
        free(w);
    }
    o_thr = thr;
    return 0;
}

static uint64_t o_poisson_key(uint64_t seed, int64_t local_id, int64_t cycle)
{
    return o_hash3(seed ^ O_POISSON_SALT, (uint64_t)local_id, (uint64_t)(cycle + 1));
}

static int32_t o_poisson_draw(uint64_t key, float rate)
{
    uint32_t q = (uint32_t)(rate * 0.015625f);
    float r = rate - (float)(q * 64u);
    float L = (float)exp(-(double)r);
    uint32_t i = 0, rest = q;
    int32_t k = 0;
    for (int l = 0; l < O_LEVELS; l++) {
        uint32_t cnt = l < O_LEVELS - 1 ? (rest & 3u) : rest;
        rest >>= 2;
        for (uint32_t c = 0; c < cnt; c++) {
            uint32_t u = (uint32_t)(o_mix64(key + (uint64_t)(i++) * 0x9e3779b97f4a7c15ULL) >> 32);
            const uint32_t *t = o_thr + o_off[l];
            int32_t idx = 0;
            while (u >= t[idx]) idx++; /* linear scan: same answer as a bisection */
            k += o_kmin[l] + idx;
        }
    }
    float p = 1.0f;
    for (;;) {
        uint32_t u24 = (uint32_t)(o_mix64(key + (uint64_t)(i++) * 0x9e3779b97f4a7c15ULL) >> 40);
        float u = ((float)u24 + 0.5f) * (1.0f / 16777216.0f);
        p = p * u;
        if (p <= L) break;
        k++;
    }
    return k;
}

/* (int)(time / dt) as the reference's reset() computes cycles, clamped to the int range. */
static int32_t o_cycle_f(float x)
{
    if (!(x < 2147483648.0f)) return INT32_MAX;
    if (x < -2147483648.0f) return INT32_MIN;
    return (int32_t)x;
}

static int32_t o_cycle_d(double x)
{
    if (!(x < 2147483648.0)) return INT32_MAX;
    if (x < -2147483648.0) return INT32_MIN;
    return (int32_t)x;
}

int oracle_poisson_draws(uint64_t seed, float rate, int64_t n, int32_t *out)
{
    if (n < 0 || (n > 0 && !out) || !(rate >= 0.0f && rate < 16777216.0f)) return -1;
    if (o_tables()) return -4;
    for (int64_t i = 0; i < n; i++) out[i] = o_poisson_draw(o_poisson_key(seed, i, -1), rate);
    return 0;
}

#define REAL float
#define SFX(name) name##_f32
#define R_EXP expf
#define R_FABS fabsf
#define R_ROUND roundf
#define R_CYCLE o_cycle_f
#include "lif_oracle_impl.h"
#undef REAL
#undef SFX
#undef R_EXP
#undef R_FABS
#undef R_ROUND
#undef R_CYCLE

#define REAL double
#define SFX(name) name##_f64
#define R_EXP exp
#define R_FABS fabs
#define R_ROUND round
#define R_CYCLE o_cycle_d
#include "lif_oracle_impl.h"
