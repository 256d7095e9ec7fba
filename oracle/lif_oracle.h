/*
 * TEST INFRASTRUCTURE ONLY — not part of the product.
 *
 * CPU restatement of BSim's single-thread simulator (STSim) for networks of
 * LIF_brian neurons (LIFENeuron) joined by StaticSynapse, used as the parity
 * oracle for the GPU engine. Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load it.
 *
 * What it restates (reference paths relative to the BSim project root):
 *   oracle_lif_reset_*  LIFENeuron::reset          src/neuron/lif/LIFENeuron.cpp:68-112
 *   oracle_syn_reset_*  StaticSynapse::reset       src/synapse/static/StaticSynapse.cpp:43-54
 *   oracle_run_*        SingleThreadSimulator::run src/sim/SingleThreadSimulator.cpp:21-183
 *                       -> Network::update         src/net/Network.cpp:308-330
 *                       -> LIFENeuron::update      src/neuron/lif/LIFENeuron.cpp:114-160
 *                       -> NeuronBase::fire        src/base/NeuronBase.cpp:47-54
 *                       -> StaticSynapse::recv/update src/synapse/static/StaticSynapse.cpp:31-70
 *                       -> LIFENeuron::recv        src/neuron/lif/LIFENeuron.cpp:52-61
 *   input-drive neurons (kind 1, 2) follow the reference's GPU kernels, whose rules
 *   differ from its CPU classes (the engine replaces SGSim):
 *                       ConstantNeuron  src/neuron/constant/constant.cu:18-22,
 *                                       reset ConstantNeuron.cpp:55-62
 *                       PoissonNeuron   src/neuron/poisson/poisson.cu:9-31,
 *                                       reset PoissonNeuron.cpp:35-44
 *   with the engine's reproducible Poisson sampler restated in lif_oracle.c (the
 *   reference's draws come from clock-seeded generators and cannot be replayed).
 *
 * Parity is pinned in tests against the reference's golden traces
 * (test/lif_unit{1..4}_test_v.std) and against the reference sources compiled
 * here (oracle/_ref, built by oracle/Makefile).
 */
#ifndef BSIM_ORACLE_H
#define BSIM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Per-neuron raw parameters, LIFENeuron constructor order:
 * v_init, v_rest, v_reset, cm, tau_m, tau_refrac, tau_syn_E, tau_syn_I, v_thresh, i_offset */
#define ORACLE_NPARAM 10
/* Folded per-neuron constants written by oracle_lif_reset_*, in this order. */
#define ORACLE_NFOLD 11 /* vm, CI, CE, C_I, C_E, v_tmp, i_I, i_E, v_thresh, v_reset, Cm */

/* Accumulation of synaptic input within one step. */
#define ORACLE_ACC_SEQUENTIAL 0 /* reference order: sequential adds in synapse creation order */
#define ORACLE_ACC_FIXED 1      /* exact int64 fixed point, quantum 2^-qexp (GPU engine default) */

typedef struct oracle_out {
    int64_t record_steps;   /* raster / trace recorded for steps [0, record_steps) */
    int32_t *fire_count;    /* [n] spikes per neuron over the whole run (may be NULL) */
    int64_t *raster_off;    /* [record_steps+1] offsets into raster_ids (may be NULL) */
    int32_t *raster_ids;    /* fired ids, ascending within a step (capacity raster_cap) */
    int64_t raster_cap;
    const int32_t *rec_ids; /* neurons whose v is traced (may be NULL) */
    int64_t n_rec;
    void *v_trace;          /* [record_steps][n_rec] REAL: v after each step's update */
    void *final_state;      /* [n][4] REAL: v, i_E, i_I, refrac_step (as REAL) at the end */
    int64_t *spikes_per_step;  /* [steps] (may be NULL) */
    int64_t *events_per_step;  /* [steps] synaptic events delivered in each step (may be NULL) */
    /* Optional square-wave drive (an input, kept here to leave the run signature
     * stable): cycle t uses the v_tmp folded from params_alt ([n][10] REAL) when
     * (t / half_period) is odd. params_alt may differ from params in i_offset only. */
    const void *params_alt;
    int64_t half_period;  /* 0: constant drive */
    /* Optional input-drive neurons (inputs as well). kind[j]: 0 LIF_brian, 1 Constant_spikes,
     * 2 Poisson_spikes (NULL = all LIF); params[j] then holds ConstantNeuron(fire_rate,
     * start_time, end_time) or PoissonNeuron(rate, refract, start_time, duration) in its
     * first slots. instance[j] (NULL = one network) and input_seed key the Poisson draws. */
    const uint8_t *kind;
    const int32_t *instance;
    uint64_t input_seed;
} oracle_out;

/* The Poisson sampler on its own: n draws of Poisson(rate), draw i keyed as the
 * initial draw of neuron id i (statistics checks). */
int oracle_poisson_draws(uint64_t seed, float rate, int64_t n, int32_t *out);

/* ---- float build (reference `real` = float) ---- */
int oracle_lif_reset_f32(const float *params, int64_t n, float dt, float *fold, int32_t *refrac_time);
int oracle_syn_reset_f32(const float *delay_s, const float *weight, const float *tau_syn,
                         int64_t s, float dt, int32_t *delay_steps, float *weight_out);
int oracle_run_f32(const float *params, int64_t n,
                   const int32_t *src, const int32_t *dst, const float *weight,
                   const int32_t *delay_steps, int64_t s, float dt, int64_t steps,
                   int acc_mode, const int32_t *qexp_per_neuron, oracle_out *out);

/* ---- double build (reference compiled with -DUSE_DOUBLE) ---- */
int oracle_lif_reset_f64(const double *params, int64_t n, double dt, double *fold, int32_t *refrac_time);
int oracle_syn_reset_f64(const double *delay_s, const double *weight, const double *tau_syn,
                         int64_t s, double dt, int32_t *delay_steps, double *weight_out);
int oracle_run_f64(const double *params, int64_t n,
                   const int32_t *src, const int32_t *dst, const double *weight,
                   const int32_t *delay_steps, int64_t s, double dt, int64_t steps,
                   int acc_mode, const int32_t *qexp_per_neuron, oracle_out *out);

#ifdef __cplusplus
}
#endif

#endif
