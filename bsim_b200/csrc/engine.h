// Internal structures of the bsim_b200 engine (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/bsim_b200.h"
#include "drive.h"

namespace bsim {

constexpr uint32_t TILE_PAD = 0xffffffffu;  // target of a padding entry of the tiled copy

// One neuron class. For LIF_brian neurons: a folded parameter tuple, the
// per-population part of LIFENeuron::reset's output (src/neuron/lif/LIFENeuron.cpp:68-112);
// v_tmp depends on i_offset and is kept per neuron. Input-drive neurons
// (BSIM_NEURON_CONSTANT / _POISSON) keep their parameters per neuron in the state
// slots and use only kind, pop, inst and id_base here. 64 bytes; the table is small
// and read through the L1 cache.
struct ClassParams {
    float Cm, CE, CI, C_E, C_I, v_thresh, v_reset;
    int32_t refrac_time;
    float scale_up;    // 2^qexp: fixed-point value of a weight is rn(w * scale_up)
    float scale_down;  // 2^-qexp
    int32_t pop;       // population (spike statistics)
    int32_t inst;      // independent network
    int32_t kind;      // BSIM_NEURON_*
    int32_t id_base;   // first neuron id of the network (Poisson draws use id - id_base)
    int32_t reserved[2];
};

// Raster recording window: cycles [t0, t0 + steps) into a buffer of cap ids.
struct RecCtl {
    long long next;   // next cycle to copy out (cycle t copies cycle t-1 once it is complete)
    long long t0;
    long long steps;  // 0: not recording
    long long cap;
};

// State trace window: after each cycle t in [t0, t0 + steps), the neurons
// [first, first + count) have v, i_E, i_I and the synaptic input the cycle
// consumed (E, I) copied into the trace buffer, field-major: [5][steps][count].
struct TraceCtl {
    long long t0;
    long long steps;  // 0: not tracing
    long long first;
    long long count;
};

// Firing-predictor statistics, accumulated on the device.
struct PredStats {
    unsigned long long cycles, fallbacks, tile_cycles;
    double abs_err, actual;
};

// Everything one fused step launch needs. Passed by value (kernel parameter space).
struct StepArgs {
    int64_t N;         // neurons
    int32_t D;         // max delay, steps
    int32_t R;         // ring slots = D + 2
    int64_t cap;       // fired ids per ring slot
    int64_t W;         // bitmap words per ring slot = ceil(N / 32)
    float4 *state;     // [N] LIF: {v, i_E, i_I, refrac_step as int bits}
                       //     Constant: {fire_rate, start_cycle, end_cycle, fire_count} (ints as bits)
                       //     Poisson: {rate, fire_cycle, end_cycle, refrac_step} (ints as bits)
    const float *vtmp; // [N] LIF: v_tmp; Poisson: exp(-(rate mod 64)); Constant: unused
    const float *vtmp_alt;  // [N] v_tmp of the odd half periods of a square-wave drive (may be NULL)
    int32_t drive_half;     // cycles per half period (0: constant drive)
    PoissonTables ptab;     // inversion tables of the Poisson sampler (NULL thr: no Poisson neurons)
    uint64_t input_seed;    // seed of the Poisson neurons' draws
    const uint16_t *cls;       // [N] class of each neuron
    const ClassParams *ctab;   // [n_cls]
    void *acc;                 // [2][n_planes][N] longlong2 (EXACT) or [2][N] float2 (ORDERED): input
                               // for the next step; a target's input is the sum over its planes
    int32_t n_planes;          // accumulator planes per parity (1 in every configuration)
    int32_t acc_clear;         // the LIF phase zeroes the planes it read (0: every cycle overwrites them)
    uint32_t *bitmap;          // [R][W] fired flags of each step in the ring
    int32_t *ring;             // [R][cap] fired ids of each step in the ring
    int32_t *ring_cnt;         // [R]
    const int64_t *row_off;    // [N*D + 1] push rows by (source, delay)
    const uint2 *syn;          // [S] {target id, weight bits}, creation order inside a row
    const int64_t *col_off;    // [N + 1] pull rows by target
    const uint32_t *csc_src;   // [S] source id, creation order inside a row
    const float *csc_w;        // [S]
    const uint8_t *csc_d;      // [S] delay - 1
    int32_t *fire_count;       // [N]
    unsigned long long *step_ctr;  // current cycle t (device-side, advanced by the last block)
    unsigned int *ticket;          // end-of-step block counter
    unsigned long long *events;    // synaptic events delivered
    int32_t *err;                  // device error flag (0 = ok)
    const int32_t *deliv_sel;      // per-step delivery choice written by the predictor (may be NULL)
    int32_t delivery;              // BSIM_DELIVERY_PUSH / _PULL when deliv_sel is NULL
    // raster recording (control words in device memory so a captured graph stays valid)
    int32_t *rec_ids;           // [rec->cap]
    int64_t *rec_off;           // [rec->steps + 1]
    struct RecCtl *rec;         // NULL: recording never enabled
    // state trace (the reference's LOG_DATA files g_v / g_ie / g_ii / g_input_e / g_input_i)
    float *trace;               // [5][trace_ctl->steps][trace_ctl->count] (NULL: never enabled)
    const struct TraceCtl *trace_ctl;
    // per-population spike counts of the last hist_len steps (predictor input)
    int32_t *pop_hist;          // [hist_len][n_pops]
    int32_t n_pops, hist_len;
    // target-tiled delivery (BSIM_DELIVERY_TILE). A tile is a target range whose
    // excitatory and inhibitory sums are formed in shared memory. Its sources form
    // runs of consecutive neuron ids; every source of a run owns one (tile, source)
    // pair. A tile's work units are split into parts, handed to blocks by a per-cycle
    // queue. A block that finds the queue empty joins the part with the most units
    // left. Every block that worked on a tile stores (the first to finish) or adds (the
    // others, once that store is done) its sums into the one accumulator plane.
    int32_t n_tiles;                 // tiles (0: no tiled copy)
    int32_t n_tiles_u;               // = n_tiles (target ranges)
    int32_t n_parts;                 // parts over all tiles
    const int4 *parts;               // [n_parts] {tile, first unit, end unit, part within the tile},
                                     // largest first
    unsigned int *part_ctr;          // next part to hand out (reset by the last block of a cycle)
    unsigned int *part_help;         // [n_parts] blocks helping each part this cycle
    unsigned int *part_next;         // [n_parts] next unit of each part: any block may take chunks
                                     // of any part (reset to the first unit by the last block)
    unsigned int *part_pairs;        // [2][n_parts] entry pairs listed per part, by cycle parity;
                                     // the previous cycle's count sizes the part's chunks
    unsigned int *tile_arrive;       // [2][n_tiles]: blocks that finished a piece of the tile this
                                     // cycle, and whether the first one's store is done (reset by
                                     // the last block)
    int32_t tile_max;                // largest range (neurons): shared-memory accumulator size
    const int32_t *tile_beg;         // [n_tiles + 1] first target of each tile
    const float *tile_scale;         // [n_tiles] 2^qexp of the tile's network
    const int32_t *tile_run_off;     // [n_tiles + 1] range of runs
    const int32_t *tile_units;       // [n_tiles] work units: sum over runs of ceil(n/32) * D
    const uint32_t *run_src0;        // [runs] first source
    const int32_t *run_n;            // [runs] sources in the run
    const int64_t *run_pair0;        // [runs] pair of the first source
    const int32_t *run_unit0;        // [runs] first work unit, counted within the tile
    const int64_t *pair_base;        // [P] first entry of each pair
    const uint16_t *pair_doff;       // [P][D + 1] cumulative entry counts by delay (padded to even)
    const uint32_t *pair_seg;        // [P][D + 1] each delay's segment start in 16-byte entry pairs,
                                     // (pair_base + pair_doff) / 2 - tile_seg0[tile]; the last one is
                                     // the pair's end
    const int64_t *tile_seg0;        // [n_tiles] first 16-byte entry pair of each tile
    const uint2 *ent;                // [E] {target within the tile, weight bits}; every (pair, delay)
                                     // segment starts on an even entry and has even length
                                     // (padding entries have target 0xffffffff)
    // firing predictor (needs pop_hist)
    const float *mlp;                // [BSIM_MLP_PARAMS] (NULL: off)
    const int32_t *pop_size;         // [n_pops]
    const float *pop_indeg;          // [n_pops] mean in-degree
    const float *pop_outdeg;         // [n_pops] mean out-degree
    float *pred_ring;                // [4][n_pops] predicted spikes of cycle s at slot s % 4
    float *pred_sum;                 // [4][2] predicted spikes and events of cycle s at slot s % 4
    PredStats *pstats;
    float pred_tol, mean_outdeg;
    float cost_push_a, cost_push_b, cost_tile_a, cost_tile_b;  // ns per cycle, ns per event
};

struct Engine {
    int device = 0;
    cudaStream_t stream = nullptr;
    bsim_options opt{};
    int sm_count = 0;
    int64_t N = 0, S = 0;
    int32_t D = 1;
    float dt = 0.0f;
    int32_t n_inst = 1, n_cls = 0, n_pops = 1;
    std::vector<int32_t> qexp;  // per instance
    int64_t steps_done = 0;
    int64_t device_bytes = 0;
    std::vector<void *> allocs;
    StepArgs a{};
    int grid = 0, block = 0;
    // CUDA graph of graph_steps fused steps
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    int graph_len = 0;
    // recording
    int64_t rec_cap_alloc = 0, rec_steps_alloc = 0;
    bool rec_dirty = false;
    int64_t trace_alloc = 0;  // floats in the trace buffer
    // read-back of the recording: the per-cycle sort's output and scratch, sized
    // when the recording is set up, so that reading allocates nothing
    int32_t *rec_sorted = nullptr;
    void *sort_tmp = nullptr;
    size_t sort_tmp_bytes = 0;
    // staging for state uploads and read-backs: four planes of N words (v, i_E,
    // i_I, refrac), so the host's arrays move with one copy each, no host repacking
    float *stage = nullptr;
    // schedule state: predictor statistics and the MLP's parameters (a.pstats / a.mlp
    // point here while a schedule / a predictor is attached)
    PredStats *pstats_mem = nullptr;
    float *mlp_mem = nullptr;
    // population statistics (device arrays in a: pop_size, pop_indeg, pop_outdeg)
    bool pop_info_ready = false;
    // tiled copy, host side: synapses and work units per tile (planning the parts)
    std::vector<int64_t> tile_entries;
    std::vector<int32_t> tile_units;
};

}  // namespace bsim
