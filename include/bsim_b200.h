/*
 * bsim_b200 — C ABI of the B200 (sm_100a) engine behind BSim's single-GPU
 * simulation step for LIF_brian neurons and static delayed synapses.
 *
 * The reference drives this path through per-type function-pointer tables
 * (src/utils/TypeFunc.h:11-21) filled with cudaAllocLIFE / cudaUpdateLIFE /
 * cudaUpdateStatic and friends, and through process-wide __device__ globals
 * (src/gpu_utils/runtime.cu:28-63). This ABI replaces those with an opaque
 * engine handle, plain pointers and sizes, and int status codes (the reference
 * calls exit() on CUDA errors, src/third_party/cuda/helper_cuda.h:985-999).
 *
 * Units are SI (V, s, F, A), as in the reference. Inhibition is a negative
 * weight. All functions return BSIM_OK (0) or a negative BSIM_ERR_* code.
 * Host pointers are plain host memory unless a name ends in _dev.
 */
#ifndef BSIM_B200_H
#define BSIM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BSIM_OK 0
#define BSIM_ERR_ARG (-1)      /* invalid argument or size */
#define BSIM_ERR_CUDA (-2)     /* CUDA runtime error (message in bsim_last_error) */
#define BSIM_ERR_DEVICE (-3)   /* device-side error flag raised (bad index, overflow, timeout) */
#define BSIM_ERR_DELAY (-4)    /* a synapse delay rounds to 0 steps or above BSIM_MAX_DELAY */
#define BSIM_ERR_NOMEM (-5)    /* device or host allocation failed */
#define BSIM_ERR_STATE (-6)    /* call not valid in the engine's current state */
#define BSIM_ERR_LIMIT (-7)    /* network exceeds a documented engine limit */

/* Codes of the device error flag (BSIM_ERR_DEVICE; the message of bsim_last_error names
 * the code). The first code raised is kept; every later cycle of the engine (or of the
 * allocation-free call) returns at once, so no cycle runs on inconsistent data. */
#define BSIM_DEVERR_ROW 1      /* a push row ends before it starts (row offsets not ascending) */
#define BSIM_DEVERR_TARGET 2   /* a synapse target outside the network */
#define BSIM_DEVERR_CLASS 3    /* a class index beyond the class table, or a class of a kind
                                  the entry point does not take */
#define BSIM_DEVERR_ROWS_END 4 /* row offsets do not start at 0 or do not end at the synapse count */
#define BSIM_DEVERR_TIMEOUT 5  /* a bounded wait inside the step ran out (the step's result is not trusted) */

#define BSIM_MAX_DELAY 1024    /* delays are 1..BSIM_MAX_DELAY steps */
#define BSIM_MAX_CLASSES 65535 /* distinct folded LIF parameter tuples per engine */

/* Neuron kinds (bsim_create_mixed). */
#define BSIM_NEURON_LIF 0      /* LIF_brian / IF_curr_exp: LIFENeuron + StaticSynapse */
#define BSIM_NEURON_CONSTANT 1 /* Constant_spikes: ConstantNeuron + StaticSynapse */
#define BSIM_NEURON_POISSON 2  /* Poisson_spikes: PoissonNeuron + StaticSynapse */

/* How one step's synaptic input is summed per target neuron. */
#define BSIM_ACC_EXACT 0   /* exact int64 fixed point (quantum 2^-qexp per network): the sum is
                              independent of delivery order, so push, pull, batched and
                              predictor-scheduled runs give bit-identical results; equal to the
                              reference's sequential fp32 sum whenever a target receives at most
                              two same-sign inputs in a step, else the correctly rounded sum. */
#define BSIM_ACC_ORDERED 1 /* sequential fp32 sums in synapse creation order, the order of the
                              reference's StaticSynapse::update loop (src/net/Network.cpp:320-325):
                              bit-identical to the reference CPU simulator. Pull delivery only. */

#define BSIM_DELIVERY_PUSH 0 /* source-ordered rows, one warp per (spike, delay) segment */
#define BSIM_DELIVERY_PULL 1 /* target-ordered rows scanned against per-step fired bitmaps */
#define BSIM_DELIVERY_AUTO 2 /* per step, by the firing predictor (EXACT accumulation only) */
#define BSIM_DELIVERY_TILE 3 /* target tiles summed in shared memory, sources filtered by their
                                fire history (EXACT accumulation only; delays up to 64) */

typedef struct bsim_engine bsim_engine;

typedef struct bsim_options {
    int32_t device;        /* CUDA device ordinal (the reference hard-codes 0, SingleGPUSimulator.cu:83) */
    int32_t accumulate;    /* BSIM_ACC_* */
    int32_t delivery;      /* BSIM_DELIVERY_* */
    int32_t build_pull;    /* also build the target-ordered copy (forced on for PULL and ORDERED) */
    int32_t graph_steps;   /* steps captured per CUDA graph by bsim_run (0: plain launches) */
    int32_t block_threads; /* threads per block of the step kernel (0: autotuned) */
    int32_t grid_blocks;   /* blocks of the step kernel (0: autotuned) */
    int32_t build_tiles;   /* 1: also build the target-tiled copy; 0: only for TILE/AUTO; -1: never
                              (an AUTO engine then pushes every cycle; saves ~8 B per synapse) */
    int32_t tile_size;     /* target neurons per tile (0: chosen from the network size and delays, <= 5000) */
    int32_t reserved[7];
} bsim_options;

/* Parameters of one generated network (see bsim_create_generated). */
typedef struct bsim_gen_spec {
    uint64_t seed;
    int32_t n_pop;         /* populations */
    int32_t pop_size;      /* neurons per population */
    float p_conn;          /* Bernoulli connection probability of each projection */
    float remote_frac;     /* fraction of populations with one extra remote projection */
    int32_t max_delay;     /* delays U{1..max_delay} steps */
    float exc_frac;        /* probability that a synapse is excitatory */
    float w_max;           /* excitatory weight U[0, w_max) */
    float inh_scale;       /* inhibitory weight -U[0, inh_scale * w_max) */
    float i_min, i_max;    /* i_offset U[i_min, i_max) per neuron */
    float v_init_lo, v_init_hi; /* v_init U[lo, hi) per neuron */
    /* LIFENeuron parameters shared by all neurons (constructor order minus v_init, i_offset) */
    float v_rest, v_reset, cm, tau_m, tau_refrac, tau_syn_E, tau_syn_I, v_thresh;
    /* Square-wave drive: in odd half periods every i_offset is multiplied by drive_scale
     * (drive_half_period cycles per half period; 0 = constant drive). */
    float drive_scale;
    int32_t drive_half_period;
} bsim_gen_spec;

typedef struct bsim_info {
    int64_t n_neurons;
    int64_t n_synapses;
    int32_t max_delay;       /* D, steps */
    int32_t n_instances;     /* independent networks packed in the engine */
    int32_t n_classes;       /* distinct folded parameter tuples */
    int32_t n_pops;          /* populations (spike statistics granularity) */
    int64_t steps_done;      /* simulated cycles so far */
    uint64_t events_total;   /* synaptic events delivered so far */
    int64_t device_bytes;    /* device memory held by the engine */
    int32_t grid_blocks, block_threads;
    int32_t accumulate, delivery;
    int32_t sm_count;
    int32_t reserved[7];
} bsim_info;

/* Fills *opt with defaults: EXACT accumulation, PUSH delivery, graphs of 64 steps. */
int bsim_options_default(bsim_options *opt);

/* Builds an engine from flat host arrays and uploads it.
 * Replaces Network::buildNetwork (src/net/BuildNetwork.cpp:36-205), copyNetworkToGPU
 * (src/gpu_utils/gpu_net_copy.cu:8-109), alloc_buffers (src/gpu_utils/GBuffers.cu:9-56),
 * the LIFE allocators cudaAllocLIFE/allocLIFE (src/neuron/lif/GLIFENeurons.cu:6,
 * GLIFENeurons.cpp:8-30) and the neuron half of Network::reset (LIFENeuron::reset,
 * src/neuron/lif/LIFENeuron.cpp:68-112, folded here in fp32 on the host exactly as there).
 *   params      [n][10] LIFENeuron constructor arguments per neuron, global id order:
 *               v_init, v_rest, v_reset, cm, tau_m, tau_refrac, tau_syn_E, tau_syn_I, v_thresh, i_offset
 *   pop         [n] population of each neuron (statistics only; may be NULL = one population)
 *   instance    [n] independent network of each neuron (may be NULL = one network); a
 *               synapse must not join two instances
 *   src, dst    [s] neuron ids, synapses in creation (Network::connect) order
 *   weight      [s] weights after StaticSynapse::reset (see bsim_synapse_reset)
 *   delay_steps [s] 1..BSIM_MAX_DELAY
 */
int bsim_create(const float *params, int64_t n, const int32_t *pop, const int32_t *instance,
                const int32_t *src, const int32_t *dst, const float *weight, const int32_t *delay_steps,
                int64_t s, float dt, const bsim_options *opt, bsim_engine **out);

/* bsim_create for networks that also hold input-drive neurons, Constant_spikes and
 * Poisson_spikes (include/Neuron.h:25-26 of the reference), stepped in the same launch
 * as the LIF neurons with the reference GPU kernels' rules:
 *   kind[i] = BSIM_NEURON_LIF       params[i] as for bsim_create
 *   kind[i] = BSIM_NEURON_CONSTANT  params[i][0..2] = ConstantNeuron(fire_rate, start_time,
 *             end_time) (src/neuron/constant/ConstantNeuron.cpp:14); fires at cycle t iff
 *             t < end_cycle and (t - start_cycle) * fire_rate > fire_count
 *             (src/neuron/constant/constant.cu:18-22), cycles = (int)(time / dt)
 *   kind[i] = BSIM_NEURON_POISSON   params[i][0..3] = PoissonNeuron(rate, refract, start_time,
 *             duration) (src/neuron/poisson/PoissonNeuron.cpp:13); fires at cycle t iff
 *             t == fire_cycle and t <= end_cycle, then fire_cycle += 1 + Poisson(rate) +
 *             (int)(refract / dt) (src/neuron/poisson/poisson.cu:9-31); the first fire_cycle is
 *             (int)(start_time / dt) + Poisson(rate); rate is the mean gap in cycles, 0..2^24.
 * The reference draws Poisson numbers from a clock-seeded host generator and curand
 * (not reproducible); here each draw is a function of (input_seed, the neuron's id minus
 * the first id of its network, the cycle), so a run is reproducible and a network gives
 * the same spikes alone or packed with others. Cycles beyond 2^31-1 are clamped to it.
 * kind may be NULL (all LIF: the same engine as bsim_create). */
int bsim_create_mixed(const float *params, const uint8_t *kind, int64_t n, const int32_t *pop,
                      const int32_t *instance, const int32_t *src, const int32_t *dst, const float *weight,
                      const int32_t *delay_steps, int64_t s, float dt, uint64_t input_seed,
                      const bsim_options *opt, bsim_engine **out);

/* Builds an engine for one or more generated networks directly on the device
 * (no host synapse arrays). Network k's neurons follow network k-1's. */
int bsim_create_generated(const bsim_gen_spec *specs, int32_t n_specs, float dt, const bsim_options *opt,
                          bsim_engine **out);

/* Host-side generator: sizes, then the flat arrays bsim_create takes, for one spec.
 * params is [n][10] in LIFENeuron constructor order. Identical to the device builder. */
int bsim_gen_count(const bsim_gen_spec *spec, int64_t *n, int64_t *s);
int bsim_gen_host(const bsim_gen_spec *spec, float *params, int32_t *pop, int32_t *src, int32_t *dst,
                  float *weight, int32_t *delay_steps);

/* StaticSynapse::reset (src/synapse/static/StaticSynapse.cpp:43-54): delays in seconds to
 * whole steps, and the weight decay exp(-(delay - dt*steps)/tau) applied when the delay is
 * not a multiple of dt. Host only. */
int bsim_synapse_reset(const float *delay_s, const float *weight, const float *tau_syn, int64_t s, float dt,
                       int32_t *delay_steps, float *weight_out);

/* Advances the simulation by `steps` cycles on the engine's stream, without host
 * synchronisation between steps; returns after the device has finished.
 * Replaces the step loop of SingleGPUSimulator::run (src/sim/SingleGPUSimulator.cu:146-245):
 * cudaUpdateLIFE (src/gpu_utils/gpu_func.cu:44-51) + cudaUpdateStatic (:67-74) +
 * update_time (src/gpu_utils/runtime.cu:81-92) fused into one launch per step. */
int bsim_run(bsim_engine *e, int64_t steps);

/* Like bsim_run but only enqueues the work (no final synchronisation). */
int bsim_run_async(bsim_engine *e, int64_t steps);
int bsim_sync(bsim_engine *e);

/* Test support for the device error path (no counterpart in the reference, whose
 * kernels have no bounded waits): marks tile `tile` of a tiled engine as already
 * claimed by a finisher of the current cycle, so every block that finishes a piece
 * of it in the next step waits for a store that never comes. The wait gives up
 * after its bound (about 0.3 s), raises BSIM_DEVERR_TIMEOUT and lets the step end;
 * bsim_run / bsim_sync then return BSIM_ERR_DEVICE and no later step runs. Every
 * access stays in bounds and the engine's buffers stay readable. BSIM_ERR_ARG
 * when the engine has no such tile. */
int bsim_stall_tile(bsim_engine *e, int32_t tile);

/* Records the fired ids of the next `max_steps` cycles into a device buffer of
 * `capacity` ids (the reference's LOG_DATA GSim.log, SingleGPUSimulator.cu:209-237,
 * without a host sync per step). Calling it again restarts the recording. */
int bsim_record(bsim_engine *e, int64_t max_steps, int64_t capacity);

/* Copies the recording out: step_off [n_steps+1], ids in step order (each step's ids
 * ascending). *n_steps receives the recorded steps. BSIM_ERR_LIMIT if the buffer overflowed. */
int bsim_read_raster(bsim_engine *e, int64_t *step_off, int32_t *ids, int64_t ids_cap, int64_t *n_steps);

/* State trace of the next `max_steps` cycles: after each cycle, v, i_E, i_I and the
 * synaptic input the cycle consumed (excitatory, inhibitory) of the neurons
 * [first, first + count) are copied into a device buffer inside the step itself — the
 * reference's LOG_DATA files g_v.data, g_ie.data, g_ii.data, g_input_e.data and
 * g_input_i.data (src/sim/SingleGPUSimulator.cu:150-206), without a host copy per cycle.
 * Calling it again restarts the trace (the buffer is kept when large enough). */
int bsim_trace(bsim_engine *e, int64_t max_steps, int64_t first, int64_t count);

/* Copies the trace out: each non-NULL array receives [n_steps][count] floats in
 * cycle order; *n_steps the cycles traced so far. */
int bsim_read_trace(bsim_engine *e, float *v, float *i_E, float *i_I, float *in_E, float *in_I, int64_t *n_steps);

/* Neuron state: v, i_E, i_I, refrac_step per neuron (cudaFetchLIFE,
 * src/neuron/lif/GLIFENeurons.cu:29-40). Any pointer may be NULL. For input-drive
 * neurons the four slots hold, as float / float bits / float bits / int:
 * Constant {fire_rate, start_cycle, end_cycle, fire_count}, Poisson {rate, fire_cycle,
 * end_cycle, refrac_step} (ints in the middle two slots as their bit patterns). */
int bsim_read_state(bsim_engine *e, float *v, float *i_E, float *i_I, int32_t *refrac_step);

/* Overwrites the neuron state from host arrays (the state half of copyNetworkToGPU,
 * src/gpu_utils/gpu_net_copy.cu:8-109, as restored by single_run). NULL leaves a field. */
int bsim_write_state(bsim_engine *e, const float *v, const float *i_E, const float *i_I, const int32_t *refrac_step);

/* The CUDA stream (cudaStream_t) all of the engine's work is enqueued on. */
int bsim_get_stream(bsim_engine *e, void **stream);

/* Square-wave drive for an engine built from arrays: in odd half periods of
 * half_period cycles, v_tmp is folded from params_hi ([n][10], normally differing
 * from the creation parameters in i_offset only). half_period = 0 turns it off. */
int bsim_set_drive(bsim_engine *e, const float *params_hi, int32_t half_period);

/* Spikes per neuron since creation (FireInfo "count", src/sim/SingleGPUSimulator.cu:263-282). */
int bsim_read_fire_count(bsim_engine *e, int32_t *count);

/* Per-population spike statistics: keeps the spike count of every population for
 * the last hist_len cycles (hist_len >= 16) in a device ring. */
int bsim_enable_pop_stats(bsim_engine *e, int32_t hist_len);

/* Spike count of each population over the last `steps` cycles ([steps][n_pops],
 * oldest first; steps <= hist_len - 2). */
int bsim_read_pop_counts(bsim_engine *e, int32_t *counts, int32_t steps);

/* Size, mean in-degree and mean out-degree of each population ([n_pops] each; any may be NULL). */
int bsim_read_pop_info(bsim_engine *e, int32_t *size, float *mean_indeg, float *mean_outdeg);

/* ---- Firing predictor -------------------------------------------------------
 * A small MLP predicts each population's rate two cycles ahead from its rates in
 * the last 8 cycles and its mean in-degree. It only steers scheduling (delivery
 * mode per cycle); it never touches the dynamics, so rasters are identical with
 * and without it. Features and target (rates are spikes / size * 10, i.e. 1.0 per
 * 1 kHz at dt = 0.1 ms): x = [r(t-1), ..., r(t-8), mean_indeg / 1000], y = r(t+1). */
#define BSIM_MLP_IN 9
#define BSIM_MLP_HIDDEN 64
#define BSIM_MLP_PARAMS (BSIM_MLP_HIDDEN * BSIM_MLP_IN + BSIM_MLP_HIDDEN + BSIM_MLP_HIDDEN * BSIM_MLP_HIDDEN + \
                         BSIM_MLP_HIDDEN + BSIM_MLP_HIDDEN + 1)
/* Parameter layout: W1[64][9], b1[64], W2[64][64], b2[64], W3[64], b3. */

/* Deterministic initialisation (uniform +-sqrt(6/(fan_in+fan_out)), zero biases). Host only. */
int bsim_mlp_init(float *params, uint64_t seed);

/* Forward pass on the GPU for n samples: x [n][9] -> y [n]. Host buffers. */
int bsim_mlp_forward(const float *params, const float *x, int64_t n, float *y);

/* Mean-squared-error loss and its gradient over n samples, on the GPU (the
 * project's own backward kernel). grad [BSIM_MLP_PARAMS]. Host buffers. */
int bsim_mlp_grad(const float *params, const float *x, const float *y_target, int64_t n, float *grad, float *loss);

/* Adam training on the GPU (mini-batches of `batch`, learning rate lr) for
 * `epochs` passes; params are read and updated in place. */
int bsim_mlp_train(float *params, const float *x, const float *y_target, int64_t n, int32_t epochs, int32_t batch,
                   float lr, uint64_t seed, float *final_loss);

/* Sets the schedule of BSIM_DELIVERY_AUTO: each cycle picks push or tiled delivery by
 * the cost models (fixed ns per cycle and ns per event of each mode, e.g. from
 * bsim_autotune or a fit over plain runs) applied to the cycle's work.
 *   params != NULL: the learned schedule (needs population statistics): the work is the
 *     predicted events of the last cycle; when a cycle's exact spike count departs from
 *     its prediction by more than tolerance (relative), its choice is recomputed from
 *     the exact count (a fallback).
 *   params == NULL with cost models: the exact schedule: the work is the exact spike
 *     count of the delivered window (the last max_delay cycles) times the mean
 *     out-degree over max_delay. A step delivers only spikes of past cycles, so its
 *     work is known before it starts.
 *   all NULL: detached; AUTO then pushes every cycle. */
int bsim_set_predictor(bsim_engine *e, const float *params, float tolerance, const float *cost_push,
                       const float *cost_tile);

typedef struct bsim_pred_stats {
    int64_t cycles;          /* cycles scheduled by the predictor */
    int64_t fallbacks;       /* cycles whose choice was recomputed from exact counts */
    int64_t tile_cycles;     /* cycles delivered with the tiled mode */
    double abs_err_sum;      /* sum over cycles and populations of |predicted - actual| spikes */
    double actual_sum;       /* sum of actual spikes over the same cycles and populations */
} bsim_pred_stats;

int bsim_predictor_stats(bsim_engine *e, bsim_pred_stats *stats);

/* Autotuner (replaces the occupancy rule of getBlockSize, src/gpu_utils/gpu_func.cu:90-127):
 * runs trial_steps cycles for each candidate (block size, grid, delivery mode) in
 * three interleaved rounds (so that every candidate sees the same drift of the
 * network's activity), keeps the one with the least summed time and reports each
 * mode's measured cost. The simulation advances by 3 x candidates x trial_steps
 * cycles (the dynamics are the same for every candidate). */
typedef struct bsim_tune_result {
    int32_t block_threads, grid_blocks, delivery;
    float best_us_per_step;
    float cost_push[2];      /* fixed ns per cycle, ns per event */
    float cost_tile[2];
    int32_t candidates;
} bsim_tune_result;

int bsim_autotune(bsim_engine *e, int32_t trial_steps, bsim_tune_result *out);

int bsim_get_info(bsim_engine *e, bsim_info *info);

/* Per-network fixed-point exponent used by BSIM_ACC_EXACT ([n_instances]). */
int bsim_get_qexp(bsim_engine *e, int32_t *qexp);

/* Frees the engine (freeGPUNetwork + free_buffers, src/gpu_utils/gpu_net_copy.cu:134-191). */
int bsim_destroy(bsim_engine *e);

/* Text of the last error raised in this thread. */
const char *bsim_last_error(void);

/* ---- Allocation-free step -------------------------------------------------
 * No counterpart in the reference: it has no entry point of this kind.
 *
 * For callers that cannot allocate device memory: a host application that owns
 * the GPU's memory through its own pool and hands its plug-ins ready-made
 * buffers (a cudaMalloc would bypass its accounting, and cudaMalloc/cudaFree can
 * synchronise the whole device), a real-time loop that cannot take an
 * allocation's latency or implicit synchronisation, or a process that has
 * already reserved the remaining device memory.
 *
 * The caller passes every input and output as device pointers; the step's
 * working memory (input accumulators, fire ring, fired bitmaps, counters) is a
 * fixed array of about 3.4 MB inside the library, held by every GPU that loads
 * the library until the process exits. Limits: n <= BSIM_NOALLOC_MAX_NEURONS,
 * max_delay <= BSIM_NOALLOC_MAX_DELAY; larger sizes return BSIM_ERR_LIMIT. No
 * cudaMalloc, cudaFree or other allocating routine is called.
 *
 * Every call looks the array's device address up (cudaGetSymbolAddress) with the
 * caller's current device, so a device reset between calls is harmless; the first
 * call on a device also sizes the launch, so make it before any stream capture.
 * All calls on a device share the array and each call clears it first: calls
 * whose GPU work overlaps (other streams, unordered threads) race on it.
 *
 * Each call runs `steps` cycles with EXACT accumulation and push delivery, on
 * `stream` (a cudaStream_t, NULL = legacy default stream), starting with no
 * spikes in flight, and returns once the work is enqueued.
 *   state_dev      [n] float4 {v, i_E, i_I, refrac_step bit pattern}, in/out, 16-byte aligned
 *   vtmp_dev       [n] (i_offset * rm + v_rest) * (1 - Cm), as LIFENeuron::reset folds it
 *   cls_dev        [n] class of each neuron, < n_classes
 *   ctab_dev       [n_classes] folded constants, scale_up = 2^qexp, scale_down = 2^-qexp,
 *                  kind = BSIM_NEURON_LIF
 *   row_off_dev    [n * max_delay + 1] rows by (source, delay - 1), delay-minor, ascending,
 *                  from 0 to n_synapses
 *   syn_dev        [2 * n_synapses] {target id < n, weight bit pattern} per entry, 16-byte aligned
 *   fire_count_dev [n] incremented by each neuron's spikes
 * Before the first cycle a check pass on the GPU reads these arrays (within the sizes
 * given) and raises the device error flag (BSIM_DEVERR_*) on a class index, kind, row
 * offset or target out of range; the cycles then do nothing. bsim_noalloc_status reads
 * the flag. Not checked: the numeric values of the state and of the folded constants,
 * and that each array really holds the number of elements stated; the arrays must not
 * change while the call's work runs. */
#define BSIM_NOALLOC_MAX_NEURONS 32768
#define BSIM_NOALLOC_MAX_DELAY 16

typedef struct bsim_class_params {
    float Cm, CE, CI, C_E, C_I, v_thresh, v_reset;
    int32_t refrac_time;
    float scale_up, scale_down;
    int32_t pop, inst;
    int32_t kind;        /* BSIM_NEURON_LIF (the only kind this entry point takes) */
    int32_t id_base;     /* 0 */
    int32_t reserved[2]; /* 0 */
} bsim_class_params;

int bsim_run_noalloc(int64_t n, int32_t max_delay, void *state_dev, const float *vtmp_dev, const uint16_t *cls_dev,
                     const bsim_class_params *ctab_dev, int32_t n_classes, const int64_t *row_off_dev,
                     const uint32_t *syn_dev, int64_t n_synapses, int32_t *fire_count_dev, int64_t steps,
                     void *stream);

/* Waits for `stream` and copies the device error flag of the most recent
 * bsim_run_noalloc call on the current device into *device_error (a host int;
 * 0 = no error, else a BSIM_DEVERR_* code). Returns BSIM_OK when the flag is 0,
 * BSIM_ERR_DEVICE when it is set. Allocates nothing. The allocation-free call's
 * companion: it has no counterpart in the reference either. */
int bsim_noalloc_status(void *stream, int32_t *device_error);

#ifdef __cplusplus
}
#endif

#endif /* BSIM_B200_H */
