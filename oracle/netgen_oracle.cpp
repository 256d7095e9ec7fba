// TEST INFRASTRUCTURE ONLY: the seeded workload generator, compiled into the
// oracle library so that the CPU baselines and the reference's own simulator
// get their networks without loading the engine library. It is the same
// header-only generator the engine's host and device builders use
// (bsim_b200/csrc/netgen.h), so the networks are identical.
#include <stdint.h>

#include "../bsim_b200/csrc/netgen.h"

namespace {
bool spec_ok(const bsim_gen_spec *g)
{
    return g && g->n_pop >= 1 && g->pop_size >= 1 && g->max_delay >= 1 && g->max_delay <= 64 &&
           (int64_t)g->n_pop * g->pop_size <= (int64_t)INT32_MAX / 2 && g->p_conn >= 0 && g->p_conn <= 1;
}
}  // namespace

extern "C" int oracle_gen_count(const bsim_gen_spec *spec, int64_t *n, int64_t *s)
{
    if (!spec_ok(spec)) return -1;
    bsim::netgen_host(*spec, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, n, s);
    return 0;
}

extern "C" int oracle_gen_host(const bsim_gen_spec *spec, float *params, int32_t *pop, int32_t *src, int32_t *dst,
                               float *weight, int32_t *delay_steps)
{
    if (!spec_ok(spec) || !src || !dst || !weight || !delay_steps) return -1;
    bsim::netgen_host(*spec, params, pop, src, dst, weight, delay_steps, nullptr, nullptr);
    return 0;
}
