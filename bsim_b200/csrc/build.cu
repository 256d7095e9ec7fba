// Engine construction (host arrays or on-device generation), the run loop and
// the C ABI entry points declared in include/bsim_b200.h.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include <cub/device/device_scan.cuh>
#include <cub/device/device_segmented_sort.cuh>

#include "engine.h"
#include "netgen.h"

namespace bsim {

cudaError_t launch_step(Engine &e);
cudaError_t launch_record_flush(Engine &e);
cudaError_t step_occupancy(int block, int accumulate, int *blocks_per_sm);
cudaError_t step_occupancy(int block, int accumulate, int *blocks_per_sm, size_t smem);
size_t step_dynamic_smem(const StepArgs &a, int block);
cudaError_t step_set_smem(int accumulate, size_t bytes);

static thread_local std::string g_err;

static int fail(int code, const std::string &msg)
{
    g_err = msg;
    return code;
}

// Lets the other translation units report through bsim_last_error().
int record_error(int code, const std::string &msg) { return fail(code, msg); }

#define CK(call)                                                                                    \
    do {                                                                                            \
        cudaError_t _e = (call);                                                                    \
        if (_e != cudaSuccess) return fail(BSIM_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(_e)); \
    } while (0)

template <typename T>
static int dalloc(Engine &e, T **p, size_t count)
{
    size_t bytes = sizeof(T) * (count ? count : 1);
    cudaError_t st = cudaMalloc((void **)p, bytes);
    if (st != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(BSIM_ERR_NOMEM, "cudaMalloc of " + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(st));
    }
    e.allocs.push_back(*p);
    e.device_bytes += (int64_t)bytes;
    return BSIM_OK;
}

#define TRY(x)                      \
    do {                            \
        int _rc = (x);              \
        if (_rc != BSIM_OK) return _rc; \
    } while (0)

// ---------------------------------------------------------------------------
// LIFENeuron::reset (src/neuron/lif/LIFENeuron.cpp:68-112), fp32, on the host
// with the C library's expf, exactly as the reference's float build folds it.
// ---------------------------------------------------------------------------
struct Folded {
    float Cm, CE, CI, C_E, C_I, v_thresh, v_reset;
    int32_t refrac_time;
    float v_tmp, v_init;
};

static Folded fold_lif(const float *p, float dt)
{
    const float ZERO = 1e-10f;  // src/utils/constant.h:20
    const float v_init = p[0], v_rest = p[1], v_reset = p[2], cm = p[3], tau_m = p[4];
    const float tau_refrac = p[5], tau_syn_E = p[6], tau_syn_I = p[7], v_thresh = p[8], i_offset = p[9];
    Folded f;
    float rm = 1.0f;
    if (fabsf(cm) > ZERO) rm = tau_m / cm;
    f.Cm = tau_m > 0 ? expf(-dt / tau_m) : 0.0f;
    f.CE = tau_syn_E > 0 ? expf(-dt / tau_syn_E) : 0.0f;
    f.CI = tau_syn_I > 0 ? expf(-dt / tau_syn_I) : 0.0f;
    float v_tmp = i_offset * rm + v_rest;
    v_tmp = v_tmp * (1.0f - f.Cm);
    float C_E = rm * tau_syn_E / (tau_syn_E - tau_m);
    float C_I = rm * tau_syn_I / (tau_syn_I - tau_m);
    f.C_E = C_E * (f.CE - f.Cm);
    f.C_I = C_I * (f.CI - f.Cm);
    f.v_thresh = v_thresh;
    f.v_reset = v_reset;
    f.refrac_time = (int32_t)(tau_refrac / dt);
    f.v_tmp = v_tmp;
    f.v_init = v_init;
    return f;
}

// Smallest k with 2^k >= x (x >= 1).
static int ceil_log2_i64(int64_t x)
{
    int k = 0;
    while (k < 63 && ((int64_t)1 << k) < x) k++;
    return k;
}

// Fixed-point exponent of one network: every per-target E or I sum of
// |w| * 2^qexp stays below 2^61, so int64 accumulation cannot overflow.
static int32_t choose_qexp(int64_t max_indeg, float max_abs_w)
{
    if (max_indeg <= 0 || !(max_abs_w > 0.0f)) return 0;
    int e_w = 0;
    frexpf(max_abs_w, &e_w);  // max_abs_w < 2^e_w
    int q = 61 - ceil_log2_i64(max_indeg) - e_w;
    if (q > 126) q = 126;
    if (q < -126) q = -126;
    return q;
}

static uint32_t f2u(float f)
{
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
}

static int finish_engine(Engine &e, const std::vector<ClassParams> &ctab);
static bool wants_tiles(const bsim_options &o, int32_t D);
static int build_tiles_host(Engine &e, const int32_t *inst, const int32_t *pop, const int32_t *src,
                            const int32_t *dst, const float *weight, const int32_t *delay, int64_t s);

static int init_device(Engine &e, const bsim_options *opt)
{
    if (opt) e.opt = *opt;
    else bsim_options_default(&e.opt);
    e.device = e.opt.device;
    CK(cudaSetDevice(e.device));
    CK(cudaDeviceGetAttribute(&e.sm_count, cudaDevAttrMultiProcessorCount, e.device));
    CK(cudaStreamCreateWithFlags(&e.stream, cudaStreamNonBlocking));
    if (e.opt.accumulate == BSIM_ACC_ORDERED) e.opt.delivery = BSIM_DELIVERY_PULL;
    if (e.opt.accumulate == BSIM_ACC_ORDERED || e.opt.delivery == BSIM_DELIVERY_PULL) e.opt.build_pull = 1;
    if (e.opt.accumulate == BSIM_ACC_ORDERED && e.opt.delivery == BSIM_DELIVERY_TILE)
        return fail(BSIM_ERR_ARG, "tiled delivery needs EXACT accumulation");
    if (e.opt.delivery == BSIM_DELIVERY_TILE && e.opt.build_tiles < 0)
        return fail(BSIM_ERR_ARG, "tiled delivery needs the tiled copy (build_tiles >= 0)");
    return BSIM_OK;
}

static void free_engine(Engine *e)
{
    if (!e) return;
    cudaSetDevice(e->device);
    if (e->graph_exec) cudaGraphExecDestroy(e->graph_exec);
    if (e->graph) cudaGraphDestroy(e->graph);
    for (void *p : e->allocs) cudaFree(p);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
}

// ---------------------------------------------------------------------------
// Host-array construction.
// ---------------------------------------------------------------------------
// (int)(time / dt) in fp32, as the reference's reset() methods compute cycles,
// clamped to the int range (the reference's cast overflows there).
static int32_t cycle_of(float time, float dt)
{
    const float c = time / dt;
    if (!(c < 2147483648.0f)) return INT32_MAX;
    if (c < -2147483648.0f) return INT32_MIN;
    return (int32_t)c;
}

static float i2f(int32_t x)
{
    float f;
    memcpy(&f, &x, 4);
    return f;
}

static int32_t clamp_i32(int64_t x) { return x > INT32_MAX ? INT32_MAX : (x < INT32_MIN ? INT32_MIN : (int32_t)x); }

static int create_from_arrays(const float *params, const uint8_t *kind, int64_t n, const int32_t *pop,
                              const int32_t *inst, const int32_t *src, const int32_t *dst, const float *weight,
                              const int32_t *delay, int64_t s, float dt, uint64_t input_seed,
                              const bsim_options *opt, Engine **out)
{
    if (!params || n <= 0 || s < 0 || (s > 0 && (!src || !dst || !weight || !delay)) || !(dt > 0) || !out)
        return fail(BSIM_ERR_ARG, "bsim_create: invalid arguments");
    for (int64_t i = 0; kind && i < n; i++) {
        if (kind[i] > BSIM_NEURON_POISSON)
            return fail(BSIM_ERR_ARG, "bsim_create: neuron " + std::to_string(i) + " has an unknown kind");
        if (kind[i] == BSIM_NEURON_POISSON && !(params[10 * i] >= 0.0f && params[10 * i] < POISSON_MAX_RATE))
            return fail(BSIM_ERR_ARG, "bsim_create: Poisson neuron " + std::to_string(i) +
                                          " has a rate outside [0, 2^24) cycles");
    }
    if (n > (int64_t)INT32_MAX - 64) return fail(BSIM_ERR_LIMIT, "bsim_create: more than 2^31-64 neurons");
    int32_t D = 1, n_inst = 1, n_pops = 1;
    for (int64_t i = 0; i < n; i++) {
        if (inst && inst[i] < 0) return fail(BSIM_ERR_ARG, "bsim_create: negative instance id");
        if (pop && pop[i] < 0) return fail(BSIM_ERR_ARG, "bsim_create: negative population id");
        if (inst) n_inst = std::max(n_inst, inst[i] + 1);
        if (pop) n_pops = std::max(n_pops, pop[i] + 1);
    }
    for (int64_t k = 0; k < s; k++) {
        if (src[k] < 0 || src[k] >= n || dst[k] < 0 || dst[k] >= n)
            return fail(BSIM_ERR_ARG, "bsim_create: synapse " + std::to_string(k) + " has a neuron id out of range");
        if (delay[k] < 1 || delay[k] > BSIM_MAX_DELAY)
            return fail(BSIM_ERR_DELAY, "bsim_create: synapse " + std::to_string(k) + " has delay " +
                                            std::to_string(delay[k]) + " steps (allowed 1.." +
                                            std::to_string(BSIM_MAX_DELAY) + ")");
        if (inst && inst[src[k]] != inst[dst[k]])
            return fail(BSIM_ERR_ARG, "bsim_create: synapse " + std::to_string(k) + " joins two instances");
        D = std::max(D, delay[k]);
    }
    // fixed-point exponent per instance
    std::vector<int64_t> indeg(n, 0);
    std::vector<float> maxw(n_inst, 0.0f);
    for (int64_t k = 0; k < s; k++) {
        indeg[dst[k]]++;
        int g = inst ? inst[dst[k]] : 0;
        maxw[g] = std::max(maxw[g], fabsf(weight[k]));
    }
    std::vector<int64_t> maxdeg(n_inst, 0);
    for (int64_t i = 0; i < n; i++) {
        int g = inst ? inst[i] : 0;
        maxdeg[g] = std::max(maxdeg[g], indeg[i]);
    }
    std::vector<int32_t> qexp(n_inst);
    for (int g = 0; g < n_inst; g++) qexp[g] = choose_qexp(maxdeg[g], maxw[g]);

    Engine *e = new Engine();
    int rc = init_device(*e, opt);
    if (rc != BSIM_OK) { free_engine(e); return rc; }
    e->N = n;
    e->S = s;
    e->D = D;
    e->dt = dt;
    e->n_inst = n_inst;
    e->n_pops = n_pops;
    e->qexp = qexp;

    // first neuron id of each network: Poisson draws are keyed by id - id_base
    std::vector<int32_t> inst_base(n_inst, INT32_MAX);
    for (int64_t i = 0; i < n; i++) {
        int g = inst ? inst[i] : 0;
        inst_base[g] = std::min(inst_base[g], (int32_t)i);
    }
    bool any_poisson = false;
    for (int64_t i = 0; kind && i < n; i++) any_poisson |= kind[i] == BSIM_NEURON_POISSON;
    std::vector<uint32_t> ptab_thr;
    PoissonTables ptab_host{};
    if (any_poisson) {
        poisson_build_tables(ptab_thr, ptab_host.off, ptab_host.len, ptab_host.kmin);
        ptab_host.thr = ptab_thr.data();
    }

    // fold and deduplicate parameter classes
    std::vector<float4> state(n);
    std::vector<float> vtmp(n);
    std::vector<uint16_t> cls(n);
    std::vector<ClassParams> ctab;
    std::map<std::vector<uint32_t>, int> cmap;
    for (int64_t i = 0; i < n; i++) {
        const int kd = kind ? kind[i] : BSIM_NEURON_LIF;
        const float *prm = params + 10 * i;
        Folded f{};
        if (kd == BSIM_NEURON_LIF) f = fold_lif(prm, dt);
        int g = inst ? inst[i] : 0;
        int pp = pop ? pop[i] : 0;
        std::vector<uint32_t> key = {(uint32_t)kd, f2u(f.Cm), f2u(f.CE), f2u(f.CI), f2u(f.C_E), f2u(f.C_I),
                                     f2u(f.v_thresh), f2u(f.v_reset), (uint32_t)f.refrac_time, (uint32_t)g,
                                     (uint32_t)pp};
        auto it = cmap.find(key);
        int c;
        if (it == cmap.end()) {
            if ((int)ctab.size() >= BSIM_MAX_CLASSES) {
                free_engine(e);
                return fail(BSIM_ERR_LIMIT, "bsim_create: more than 65535 distinct LIF parameter classes");
            }
            ClassParams cp{};
            cp.Cm = f.Cm; cp.CE = f.CE; cp.CI = f.CI; cp.C_E = f.C_E; cp.C_I = f.C_I;
            cp.v_thresh = f.v_thresh; cp.v_reset = f.v_reset; cp.refrac_time = f.refrac_time;
            cp.scale_up = ldexpf(1.0f, qexp[g]);
            cp.scale_down = ldexpf(1.0f, -qexp[g]);
            cp.pop = pp;
            cp.inst = g;
            cp.kind = kd;
            cp.id_base = inst_base[g];
            c = (int)ctab.size();
            ctab.push_back(cp);
            cmap.emplace(key, c);
        } else {
            c = it->second;
        }
        cls[i] = (uint16_t)c;
        if (kd == BSIM_NEURON_LIF) {
            vtmp[i] = f.v_tmp;
            state[i] = make_float4(f.v_init, 0.0f, 0.0f, 0.0f);  // refrac_step = 0 (int bits 0)
        } else if (kd == BSIM_NEURON_CONSTANT) {
            // ConstantNeuron::reset (src/neuron/constant/ConstantNeuron.cpp:55-62)
            vtmp[i] = 0.0f;
            state[i] = make_float4(prm[0], i2f(cycle_of(prm[1], dt)), i2f(cycle_of(prm[2], dt)), i2f(0));
        } else {
            // PoissonNeuron::reset (src/neuron/poisson/PoissonNeuron.cpp:35-44); endTime = start + duration
            const float rate = prm[0];
            const uint32_t q = (uint32_t)(rate * 0.015625f);
            const float r = rate - (float)(q * 64u);
            const float exp_neg_r = (float)exp(-(double)r);
            const int32_t start = cycle_of(prm[2], dt);
            const int32_t end = cycle_of(prm[2] + prm[3], dt);
            const int32_t rs = cycle_of(prm[1], dt);
            const int32_t first = poisson_draw(poisson_key(input_seed, i - inst_base[g], -1), rate, exp_neg_r, ptab_host);
            vtmp[i] = exp_neg_r;
            state[i] = make_float4(rate, i2f(clamp_i32((int64_t)start + first)), i2f(end), i2f(rs));
        }
    }
    e->n_cls = (int)ctab.size();

    // push rows: counting sort by (source, delay), creation order kept inside a row
    // (the order of BuildNetwork.cpp:96-136)
    const int64_t nrows = n * (int64_t)D;
    std::vector<int64_t> row_off(nrows + 1, 0);
    for (int64_t k = 0; k < s; k++) row_off[(int64_t)src[k] * D + delay[k] - 1 + 1]++;
    for (int64_t r = 0; r < nrows; r++) row_off[r + 1] += row_off[r];
    std::vector<uint2> syn(s > 0 ? s : 1);
    {
        std::vector<int64_t> cur(row_off.begin(), row_off.end() - 1);
        for (int64_t k = 0; k < s; k++) {
            int64_t at = cur[(int64_t)src[k] * D + delay[k] - 1]++;
            syn[at] = make_uint2((uint32_t)dst[k], f2u(weight[k]));
        }
    }
    StepArgs &a = e->a;
    a.N = n;
    a.D = D;
    float4 *d_state;
    float *d_vtmp;
    uint16_t *d_cls;
    int64_t *d_row;
    uint2 *d_syn;
    if ((rc = dalloc(*e, &d_state, n)) || (rc = dalloc(*e, &d_vtmp, n)) || (rc = dalloc(*e, &d_cls, n)) ||
        (rc = dalloc(*e, &d_row, nrows + 1)) || (rc = dalloc(*e, &d_syn, s))) {
        free_engine(e);
        return rc;
    }
    cudaMemcpy(d_state, state.data(), sizeof(float4) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(d_vtmp, vtmp.data(), sizeof(float) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(d_cls, cls.data(), sizeof(uint16_t) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(d_row, row_off.data(), sizeof(int64_t) * (nrows + 1), cudaMemcpyHostToDevice);
    if (s > 0) cudaMemcpy(d_syn, syn.data(), sizeof(uint2) * s, cudaMemcpyHostToDevice);
    a.state = d_state;
    a.vtmp = d_vtmp;
    a.cls = d_cls;
    a.row_off = d_row;
    a.syn = d_syn;
    std::vector<uint2>().swap(syn);
    a.input_seed = input_seed;
    if (any_poisson) {
        uint32_t *d_thr;
        if ((rc = dalloc(*e, &d_thr, (int64_t)ptab_thr.size()))) {
            free_engine(e);
            return rc;
        }
        cudaMemcpy(d_thr, ptab_thr.data(), sizeof(uint32_t) * ptab_thr.size(), cudaMemcpyHostToDevice);
        a.ptab = ptab_host;
        a.ptab.thr = d_thr;
    }

    if (e->opt.build_pull) {
        // pull rows: counting sort by target, creation order kept inside a row
        std::vector<int64_t> col_off(n + 1, 0);
        for (int64_t k = 0; k < s; k++) col_off[dst[k] + 1]++;
        for (int64_t i = 0; i < n; i++) col_off[i + 1] += col_off[i];
        std::vector<uint32_t> csrc(s > 0 ? s : 1);
        std::vector<float> cw(s > 0 ? s : 1);
        std::vector<uint8_t> cd(s > 0 ? s : 1);
        if (D > 256) {
            free_engine(e);
            return fail(BSIM_ERR_LIMIT, "bsim_create: pull delivery supports delays up to 256 steps");
        }
        std::vector<int64_t> cur(col_off.begin(), col_off.end() - 1);
        for (int64_t k = 0; k < s; k++) {
            int64_t at = cur[dst[k]]++;
            csrc[at] = (uint32_t)src[k];
            cw[at] = weight[k];
            cd[at] = (uint8_t)(delay[k] - 1);
        }
        int64_t *d_col;
        uint32_t *d_csrc;
        float *d_cw;
        uint8_t *d_cd;
        if ((rc = dalloc(*e, &d_col, n + 1)) || (rc = dalloc(*e, &d_csrc, s)) || (rc = dalloc(*e, &d_cw, s)) ||
            (rc = dalloc(*e, &d_cd, s))) {
            free_engine(e);
            return rc;
        }
        cudaMemcpy(d_col, col_off.data(), sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice);
        if (s > 0) {
            cudaMemcpy(d_csrc, csrc.data(), sizeof(uint32_t) * s, cudaMemcpyHostToDevice);
            cudaMemcpy(d_cw, cw.data(), sizeof(float) * s, cudaMemcpyHostToDevice);
            cudaMemcpy(d_cd, cd.data(), s, cudaMemcpyHostToDevice);
        }
        a.col_off = d_col;
        a.csc_src = d_csrc;
        a.csc_w = d_cw;
        a.csc_d = d_cd;
    }
    cudaError_t st = cudaGetLastError();
    if (st != cudaSuccess) {
        free_engine(e);
        return fail(BSIM_ERR_CUDA, std::string("bsim_create upload: ") + cudaGetErrorString(st));
    }
    if (wants_tiles(e->opt, D)) {
        rc = build_tiles_host(*e, inst, pop, src, dst, weight, delay, s);
        if (rc != BSIM_OK) {
            free_engine(e);
            return rc;
        }
    }
    rc = finish_engine(*e, ctab);
    if (rc != BSIM_OK) {
        free_engine(e);
        return rc;
    }
    *out = e;
    return BSIM_OK;
}

#ifndef MAX_PLANES
#define MAX_PLANES 8  // parts per tile at most
#endif
#ifndef TILE_PARTS_PER_SM
#define TILE_PARTS_PER_SM 3.4  // parts over all tiles per SM, about two per resident block (measured:
                               // 2 parts per tile on 300 tiles and 3 on 148 tiles beat 1 / 4 and 4)
#endif
#ifndef MIN_PLANES
#define MIN_PLANES 1  // parts per tile at least (blocks that run out of parts help the others)
#endif

// Ring, bitmaps, accumulators, counters; launch shape. Shared by both builders.
static int finish_engine(Engine &e, const std::vector<ClassParams> &ctab)
{
    StepArgs &a = e.a;
    a.N = e.N;
    a.D = e.D;
    a.R = e.D + 2;
    a.cap = e.N;
    a.W = (e.N + 31) / 32;
    ClassParams *d_ctab;
    TRY(dalloc(e, &d_ctab, ctab.size()));
    CK(cudaMemcpy(d_ctab, ctab.data(), sizeof(ClassParams) * ctab.size(), cudaMemcpyHostToDevice));
    a.ctab = d_ctab;
    // tiled delivery: each tile's work units in P parts (TILE_PARTS_PER_SM parts per SM
    // over all tiles, MIN_PLANES..MAX_PLANES per tile); all parts of a tile (and the
    // blocks helping them) sum into one accumulator plane: the first to finish stores
    // its sums, the others add theirs once that store is done. One plane per parity for
    // every delivery mode (the step kernel keeps the plane count a runtime value: with
    // the count folded away its code generation measured 1-15 % slower)
    a.n_planes = 1;
    a.n_parts = 0;
    a.parts = nullptr;
    a.part_next = nullptr;
    a.part_pairs = nullptr;
    a.tile_arrive = nullptr;
    if (a.n_tiles > 0) {
        const int nt = a.n_tiles;
        const double want = (double)TILE_PARTS_PER_SM * e.sm_count / nt;
        const int P = (int)std::max((double)MIN_PLANES, std::min((double)MAX_PLANES, std::floor(want + 0.5)));
        unsigned int *d_arrive;
        TRY(dalloc(e, &d_arrive, 2 * (size_t)nt));  // [2][n_tiles]: finishers so far, first store done
        CK(cudaMemset(d_arrive, 0, sizeof(unsigned int) * 2 * nt));
        a.tile_arrive = d_arrive;
        std::vector<int4> parts;
        for (int q = 0; q < nt; q++) {
            const int U = q < (int)e.tile_units.size() ? e.tile_units[q] : 0;
            for (int k = 0; k < P; k++)
                parts.push_back(make_int4(q, (int)((int64_t)U * k / P), (int)((int64_t)U * (k + 1) / P), k));
        }
        // largest expected work first, so the queue ends with small parts
        std::stable_sort(parts.begin(), parts.end(), [&](const int4 &x, const int4 &y) {
            const int64_t ex = x.x < (int)e.tile_entries.size() ? e.tile_entries[x.x] : 0;
            const int64_t ey = y.x < (int)e.tile_entries.size() ? e.tile_entries[y.x] : 0;
            return ex > ey;
        });
        int4 *d_parts;
        unsigned int *d_next;
        std::vector<unsigned int> next(parts.size());
        for (size_t i = 0; i < parts.size(); i++) next[i] = (unsigned)parts[i].y;
        TRY(dalloc(e, &d_parts, parts.size()));
        TRY(dalloc(e, &d_next, parts.size()));
        CK(cudaMemcpy(d_parts, parts.data(), sizeof(int4) * parts.size(), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d_next, next.data(), sizeof(unsigned int) * parts.size(), cudaMemcpyHostToDevice));
        unsigned int *d_help;
        TRY(dalloc(e, &d_help, parts.size()));
        CK(cudaMemset(d_help, 0, sizeof(unsigned int) * parts.size()));
        a.part_help = d_help;
        unsigned int *d_pairs;
        TRY(dalloc(e, &d_pairs, 2 * parts.size()));
        CK(cudaMemset(d_pairs, 0, sizeof(unsigned int) * 2 * parts.size()));
        a.part_pairs = d_pairs;
        a.parts = d_parts;
        a.part_next = d_next;
        a.n_parts = (int32_t)parts.size();
    }
    const size_t acc_elem = e.opt.accumulate == BSIM_ACC_ORDERED ? sizeof(float2) : sizeof(longlong2);
    const size_t acc_count = 2 * (size_t)a.n_planes * (size_t)e.N;
    char *d_acc;
    TRY(dalloc(e, &d_acc, acc_elem * acc_count));
    CK(cudaMemset(d_acc, 0, acc_elem * acc_count));
    a.acc = d_acc;
    uint32_t *d_bm;
    TRY(dalloc(e, &d_bm, (size_t)a.R * a.W));
    CK(cudaMemset(d_bm, 0, sizeof(uint32_t) * (size_t)a.R * a.W));
    a.bitmap = d_bm;
    int32_t *d_ring, *d_ring_cnt, *d_fc, *d_err;
    TRY(dalloc(e, &d_ring, (size_t)a.R * a.cap));
    TRY(dalloc(e, &d_ring_cnt, a.R));
    CK(cudaMemset(d_ring_cnt, 0, sizeof(int32_t) * a.R));
    TRY(dalloc(e, &d_fc, e.N));
    CK(cudaMemset(d_fc, 0, sizeof(int32_t) * e.N));
    TRY(dalloc(e, &d_err, 1));
    CK(cudaMemset(d_err, 0, sizeof(int32_t)));
    a.ring = d_ring;
    a.ring_cnt = d_ring_cnt;
    a.fire_count = d_fc;
    a.err = d_err;
    unsigned long long *d_ctr;
    TRY(dalloc(e, &d_ctr, 4));
    CK(cudaMemset(d_ctr, 0, sizeof(unsigned long long) * 4));
    a.step_ctr = d_ctr;
    a.events = d_ctr + 1;
    a.ticket = reinterpret_cast<unsigned int *>(d_ctr + 2);
    a.part_ctr = reinterpret_cast<unsigned int *>(d_ctr + 3);
    a.delivery = (e.opt.delivery == BSIM_DELIVERY_PULL || e.opt.delivery == BSIM_DELIVERY_AUTO) ? e.opt.delivery
                                                                                                 : BSIM_DELIVERY_PUSH;
    a.deliv_sel = nullptr;
    a.rec_ids = nullptr;
    a.rec_off = nullptr;
    a.rec = nullptr;
    a.pop_hist = nullptr;
    a.n_pops = e.n_pops;
    a.hist_len = 0;
    if (a.n_tiles > 0 && e.opt.delivery == BSIM_DELIVERY_TILE) a.delivery = BSIM_DELIVERY_TILE;
    // every cycle of a tiled-only engine overwrites all planes of the parity it
    // delivers into, so the LIF phase need not clear them; any other mode adds
    a.acc_clear = a.delivery == BSIM_DELIVERY_TILE ? 0 : 1;
    // launch shape: all blocks resident (occupancy-sized grid), so the grid-stride
    // loops of both phases see every SM
    e.block = e.opt.block_threads > 0 ? e.opt.block_threads : 512;
    if (e.block % 32 != 0 || e.block > 512) return fail(BSIM_ERR_ARG, "block_threads must be a multiple of 32 <= 512");
    const size_t smem = step_dynamic_smem(a, e.block);
    if (smem > 0) CK(step_set_smem(e.opt.accumulate, smem));
    int bps = 0;
    CK(step_occupancy(e.block, e.opt.accumulate, &bps, smem));
    if (bps < 1) return fail(BSIM_ERR_LIMIT, "step kernel does not fit on an SM with this tile size");
    e.grid = e.opt.grid_blocks > 0 ? e.opt.grid_blocks : e.sm_count * bps;
    CK(cudaDeviceSynchronize());
    return BSIM_OK;
}

// Target tiles: contiguous neuron ranges that never straddle two networks, of
// near-equal size <= tile (so one shared-memory accumulator array fits them).
static int plan_tiles(const std::vector<int64_t> &run_beg, int64_t tile, std::vector<int32_t> &tile_beg,
                      int32_t &tile_max)
{
    tile_beg.clear();
    tile_max = 0;
    for (size_t r = 0; r + 1 < run_beg.size(); r++) {
        const int64_t b = run_beg[r], len = run_beg[r + 1] - b;
        if (len <= 0) continue;
        const int64_t k = (len + tile - 1) / tile;
        for (int64_t i = 0; i < k; i++) {
            const int64_t s0 = b + len * i / k, s1 = b + len * (i + 1) / k;
            tile_beg.push_back((int32_t)s0);
            tile_max = std::max<int32_t>(tile_max, (int32_t)(s1 - s0));
        }
    }
    tile_beg.push_back((int32_t)run_beg.back());
    return BSIM_OK;
}

// 16 bytes of shared counters per target (two words per E and I sum): tiles of
// <= 5000 targets let two 512-thread blocks share an SM. Every tile scans the
// fire bitmaps of its sources for each delay (a cost of tiles x D), while a
// source's segment into a tile shrinks with the tile; blocks that run out of
// parts help the others, so a few hundred tiles balance the GPU. Measured on the
// generator's networks at their steady rates: ~300 tiles of ~3,300 targets best for
// 1e6 neurons at D = 6 (7 % faster than 400 of 2,500), 5,000 targets for 2e6
// neurons, ~1,700 targets at D = 6 for smaller ones, >= 5,000 at D = 50: so the
// larger of N / (2 x SMs) and 1,700 x sqrt(D / 6), and small networks are cut
// into at least SMs / 2 tiles (the parts split them further).
static int64_t auto_tile_size(const bsim_options &o, int64_t N, int sm_count, int32_t D)
{
    if (o.tile_size > 0) return std::min<int64_t>(o.tile_size, 12288);
    int64_t t = std::max<int64_t>((int64_t)std::ceil((double)N / (2.0 * sm_count)),
                                  (int64_t)(1700.0 * std::sqrt((double)D / 6.0)));
    t = std::min<int64_t>(t, (2 * N + sm_count - 1) / sm_count);
    return std::max<int64_t>(256, std::min<int64_t>(5000, t));
}

static bool wants_tiles(const bsim_options &o, int32_t D)
{
    return o.accumulate == BSIM_ACC_EXACT && D <= 64 && o.build_tiles >= 0 &&
           (o.build_tiles > 0 || o.delivery == BSIM_DELIVERY_TILE || o.delivery == BSIM_DELIVERY_AUTO);
}

// Host-side description of the tiled copy.
struct TileHost {
    int32_t n_u = 0;  // tiles (target ranges)
    std::vector<int32_t> tile_beg, tile_run_off, tile_units, run_n, run_unit0;
    std::vector<float> tile_scale;
    std::vector<uint32_t> run_src0;
    std::vector<int64_t> run_pair0;
    int32_t tile_max = 0;
};

// Appends a run of sources [src0, src0 + n) to tile q (the last tile so far).
static void add_run(TileHost &th, uint32_t src0, int32_t n, int64_t pair0, int32_t D)
{
    const int32_t q = (int32_t)th.tile_units.size() - 1;
    th.run_src0.push_back(src0);
    th.run_n.push_back(n);
    th.run_pair0.push_back(pair0);
    th.run_unit0.push_back(th.tile_units[q]);
    th.tile_units[q] += ((n + 31) / 32) * D;
    th.tile_run_off[q + 1] = (int32_t)th.run_src0.size();
}

// Uploads the tile tables (pair and entry arrays are uploaded by the caller)
// and points the step arguments at them.
static int upload_tiles(Engine &e, const TileHost &th)
{
    StepArgs &a = e.a;
    const int32_t nt = (int32_t)th.tile_scale.size();
    const size_t nr = th.run_src0.size();
    int32_t *d_tb, *d_tro, *d_tu, *d_rn, *d_ru;
    float *d_ts;
    uint32_t *d_rs;
    int64_t *d_rp;
    TRY(dalloc(e, &d_tb, th.n_u + 1));
    TRY(dalloc(e, &d_ts, nt));
    TRY(dalloc(e, &d_tro, nt + 1));
    TRY(dalloc(e, &d_tu, nt));
    TRY(dalloc(e, &d_rs, nr));
    TRY(dalloc(e, &d_rn, nr));
    TRY(dalloc(e, &d_rp, nr));
    TRY(dalloc(e, &d_ru, nr));
    CK(cudaMemcpy(d_tb, th.tile_beg.data(), 4 * (th.n_u + 1), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_ts, th.tile_scale.data(), 4 * nt, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_tro, th.tile_run_off.data(), 4 * (nt + 1), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_tu, th.tile_units.data(), 4 * nt, cudaMemcpyHostToDevice));
    if (nr) {
        CK(cudaMemcpy(d_rs, th.run_src0.data(), 4 * nr, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d_rn, th.run_n.data(), 4 * nr, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d_rp, th.run_pair0.data(), 8 * nr, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d_ru, th.run_unit0.data(), 4 * nr, cudaMemcpyHostToDevice));
    }
    a.n_tiles = nt;
    a.n_tiles_u = th.n_u;
    e.tile_units = th.tile_units;
    a.tile_max = th.tile_max;
    a.tile_beg = d_tb;
    a.tile_scale = d_ts;
    a.tile_run_off = d_tro;
    a.tile_units = d_tu;
    a.run_src0 = d_rs;
    a.run_n = d_rn;
    a.run_pair0 = d_rp;
    a.run_unit0 = d_ru;
    return BSIM_OK;
}

// Segment starts of every (pair, delay) in 16-byte entry pairs, relative to the
// first entry pair of the pair's tile (so each tile, not the whole copy, must
// stay below 2^32 entry pairs), from the pair offsets and the per-delay
// cumulative counts (all even).
__global__ void tile_seg0_kernel(const int64_t *pair_base, const int64_t *tile_pair0, int32_t nt, int64_t n_pairs,
                                 int64_t *tile_seg0)
{
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nt; q += gridDim.x * blockDim.x)
        tile_seg0[q] = tile_pair0[q] < n_pairs ? (pair_base[tile_pair0[q]] >> 1) : 0;
}

__global__ void pair_seg_kernel(const int64_t *pair_base, const uint16_t *pair_doff, int64_t n_pairs, int D,
                                const int64_t *tile_pair0, int32_t nt, const int64_t *tile_seg0, uint32_t *pair_seg)
{
    const int64_t n = n_pairs * (D + 1);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = i / (D + 1);
        int lo = 0, hi = nt - 1;  // the tile whose pair range holds k
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (tile_pair0[mid] <= k) lo = mid;
            else hi = mid - 1;
        }
        pair_seg[i] = (uint32_t)(((pair_base[k] + pair_doff[i]) >> 1) - tile_seg0[lo]);
    }
}

// Entry order inside each (pair, delay) segment of the tiled copy. The sums do
// not depend on it (exact integers), but the step's shared-memory additions do:
// a warp adds the first entries of 32 consecutive 16-byte pairs in one atomic
// instruction and the second entries in the next, and lanes whose counters share
// a bank serialise. Each segment of up to TILE_SPREAD_MAX entries is reordered so
// that its first entries (even positions) and its second entries (odd positions)
// each cycle through distinct banks: every bank's entries are split between the
// two halves, and each half is laid out bank by bank in rounds. The counter word
// of an entry is its target (E) or 2 x tile size + target (I), so the bank is
// that index mod 32. A padding entry stays last (the second entry of its pair).
#ifndef TILE_BANK_SPREAD
#define TILE_BANK_SPREAD 1
#endif
#define TILE_SPREAD_MAX 256
#define SPREAD_WARPS 8

static __device__ __forceinline__ int entry_bank(uint2 v, int T)
{
    const float w = __uint_as_float(v.y);
    return (int)((v.x + (w >= 0.0f ? 0u : 2u * (unsigned)T)) & 31u);
}

// One warp per (tile, source) pair, the lanes working on one segment at a time:
// each entry takes a rank within its bank (shared-memory atomics, so the order
// inside a bank is arbitrary: it changes nothing), lane b splits bank b's entries
// between the halves, and each entry computes its place from the 32 banks' counts.
__global__ void __launch_bounds__(32 * SPREAD_WARPS) tile_spread_kernel(uint2 *ent, const int64_t *pair_base,
                                                                      const uint16_t *pair_doff, int64_t n_pairs,
                                                                      int D, const int64_t *tile_pair0,
                                                                      const int32_t *tile_size, int32_t nt)
{
    __shared__ uint8_t s_bank[SPREAD_WARPS][TILE_SPREAD_MAX];
    __shared__ uint16_t s_rank[SPREAD_WARPS][TILE_SPREAD_MAX];
    __shared__ uint16_t s_perm[SPREAD_WARPS][TILE_SPREAD_MAX];
    __shared__ int s_cnt[SPREAD_WARPS][32], s_ne[SPREAD_WARPS][32];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    uint8_t *bank = s_bank[wib];
    uint16_t *rank = s_rank[wib], *perm = s_perm[wib];
    int *cnt = s_cnt[wib], *nes = s_ne[wib];
    for (int64_t k = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < n_pairs;
         k += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        int lo = 0, hi = nt - 1;  // the tile whose pair range holds k
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (tile_pair0[mid] <= k) lo = mid;
            else hi = mid - 1;
        }
        const int T = tile_size[lo];
        for (int d = 0; d < D; d++) {
            const int64_t b0 = pair_base[k] + pair_doff[k * (D + 1) + d];
            const int L = (int)(pair_doff[k * (D + 1) + d + 1] - pair_doff[k * (D + 1) + d]);
            if (L <= 2 || L > TILE_SPREAD_MAX) continue;  // nothing to spread, or kept in target order
            const int pad = ent[b0 + L - 1].x == TILE_PAD ? 1 : 0;
            const int nreal = L - pad, half = L / 2;
            cnt[lane] = 0;
            __syncwarp();
            for (int i = lane; i < nreal; i += 32) {
                const int bk = entry_bank(ent[b0 + i], T);
                bank[i] = (uint8_t)bk;
                rank[i] = (uint16_t)atomicAdd(&cnt[bk], 1);
            }
            __syncwarp();
            // lane b: how many of bank b's entries go to the first half; banks with an odd
            // count give their extra entry to the first half while it is short
            const int c = cnt[lane];
            int floors = c >> 1;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) floors += __shfl_xor_sync(0xffffffffu, floors, o);
            const unsigned odd = __ballot_sync(0xffffffffu, c & 1);
            const int extra = half - floors;
            nes[lane] = (c >> 1) + (((c & 1) && __popc(odd & ((1u << lane) - 1u)) < extra) ? 1 : 0);
            __syncwarp();
            // each half in rounds over the banks: an entry of rank r in its bank's share of a
            // half goes after every entry of lower rounds and after round r's lower banks
            for (int i = lane; i < nreal; i += 32) {
                const int bk = bank[i];
                const int ne = nes[bk];
                const bool first = rank[i] < ne;
                const int r = first ? rank[i] : rank[i] - ne;
                int pos = 0;
                for (int b = 0; b < 32; b++) {
                    const int share = first ? nes[b] : cnt[b] - nes[b];
                    pos += min(share, r) + ((b < bk && share > r) ? 1 : 0);
                }
                perm[first ? 2 * pos : 2 * pos + 1] = (uint16_t)i;
            }
            if (pad && lane == 0) perm[L - 1] = (uint16_t)(L - 1);
            __syncwarp();
            // gather through registers, then store in place
            uint2 outv[TILE_SPREAD_MAX / 32];
            for (int i = lane, j = 0; i < L; i += 32, j++) outv[j] = ent[b0 + perm[i]];
            __syncwarp();
            for (int i = lane, j = 0; i < L; i += 32, j++) ent[b0 + i] = outv[j];
            __syncwarp();
        }
    }
}

// tile_pair0: [nt + 1] first pair of each tile (pairs are grouped by tile); tile_beg: [nt + 1]
// first target of each tile.
static int make_pair_seg(Engine &e, int64_t n_pairs, const std::vector<int64_t> &tile_pair0,
                         const std::vector<int32_t> &tile_beg)
{
    const int32_t nt = (int32_t)tile_pair0.size() - 1;
    for (int32_t q = 0; q < nt && q < (int32_t)e.tile_entries.size(); q++)
        if (e.tile_entries[q] / 2 > (int64_t)UINT32_MAX)
            return fail(BSIM_ERR_LIMIT, "tiled delivery: a tile with more than 2^33 entries");
    uint32_t *d_seg;
    int64_t *d_seg0, *d_tp0;
    TRY(dalloc(e, &d_seg, (size_t)n_pairs * (e.D + 1)));
    TRY(dalloc(e, &d_seg0, std::max<int32_t>(nt, 1)));
    TRY(dalloc(e, &d_tp0, nt + 1));
    CK(cudaMemcpy(d_tp0, tile_pair0.data(), sizeof(int64_t) * (nt + 1), cudaMemcpyHostToDevice));
    if (nt > 0) tile_seg0_kernel<<<e.sm_count, 256, 0, e.stream>>>(e.a.pair_base, d_tp0, nt, n_pairs, d_seg0);
    if (n_pairs > 0 && nt > 0)
        pair_seg_kernel<<<e.sm_count * 4, 256, 0, e.stream>>>(e.a.pair_base, e.a.pair_doff, n_pairs, e.D, d_tp0, nt,
                                                             d_seg0, d_seg);
    if (TILE_BANK_SPREAD && n_pairs > 0 && nt > 0) {
        std::vector<int32_t> size(nt);
        for (int32_t q = 0; q < nt; q++) size[q] = tile_beg[q + 1] - tile_beg[q];
        int32_t *d_size;
        TRY(dalloc(e, &d_size, nt));
        CK(cudaMemcpy(d_size, size.data(), sizeof(int32_t) * nt, cudaMemcpyHostToDevice));
        tile_spread_kernel<<<e.sm_count * 8, 32 * SPREAD_WARPS, 0, e.stream>>>(
            const_cast<uint2 *>(e.a.ent), e.a.pair_base, e.a.pair_doff, n_pairs, e.D, d_tp0, d_size, nt);
    }
    CK(cudaStreamSynchronize(e.stream));
    CK(cudaGetLastError());
    e.a.pair_seg = d_seg;
    e.a.tile_seg0 = d_seg0;
    return BSIM_OK;
}

// Host construction of the tiled copy: target ranges follow population (and
// network) boundaries; synapses sorted by (tile of the target, source, delay);
// one pair per distinct (tile, source), runs of consecutive sources.
static int build_tiles_host(Engine &e, const int32_t *inst, const int32_t *pop, const int32_t *src,
                            const int32_t *dst, const float *weight, const int32_t *delay, int64_t s)
{
    const int64_t n = e.N;
    const int32_t D = e.D;
    std::vector<int64_t> runs = {0};
    for (int64_t i = 1; i < n; i++)
        if ((inst && inst[i] != inst[i - 1]) || (pop && pop[i] != pop[i - 1])) runs.push_back(i);
    runs.push_back(n);
    TileHost th;
    plan_tiles(runs, auto_tile_size(e.opt, n, e.sm_count, D), th.tile_beg, th.tile_max);
    th.n_u = (int32_t)th.tile_beg.size() - 1;
    const int32_t nu = th.n_u, nt = nu;
    std::vector<int32_t> tile_of(n);
    for (int32_t q = 0; q < nu; q++)
        for (int64_t i = th.tile_beg[q]; i < th.tile_beg[q + 1]; i++) tile_of[i] = q;
    // tile (< 2^27) | source (< 2^31) | delay - 1 (< 64)
    std::vector<std::pair<uint64_t, int64_t>> key(s);
    for (int64_t k = 0; k < s; k++) {
        const uint64_t q = (uint64_t)tile_of[dst[k]];
        key[k] = {(q << 37) | ((uint64_t)src[k] << 6) | (uint64_t)(delay[k] - 1), k};
    }
    std::sort(key.begin(), key.end());
    th.tile_scale.resize(nt);
    for (int32_t q = 0; q < nt; q++) th.tile_scale[q] = ldexpf(1.0f, e.qexp[inst ? inst[th.tile_beg[q]] : 0]);
    th.tile_run_off.assign(nt + 1, 0);
    // a tile scans the delay slots of its own network's longest delay only, so
    // networks with short delays packed beside long-delay ones do not pay for them
    std::vector<int32_t> dmax_inst(std::max<int32_t>(1, e.n_inst), 1);
    for (int64_t k = 0; k < s; k++) {
        int32_t &dm = dmax_inst[inst ? inst[src[k]] : 0];
        dm = std::max(dm, delay[k]);
    }
    auto tile_D = [&](int32_t q) { return dmax_inst[inst ? inst[th.tile_beg[q]] : 0]; };
    std::vector<int64_t> pair_base;
    std::vector<uint16_t> pair_doff;
    std::vector<uint2> ent;
    ent.reserve((size_t)s + (size_t)s / 8 + 16);
    const uint2 pad = make_uint2(TILE_PAD, TILE_PAD);
    std::vector<int64_t> cnt(D);
    int32_t cur_d = -1;
    auto close_group = [&]() {  // pads the current (pair, delay) segment to even length
        if (cur_d >= 0 && (cnt[cur_d] & 1)) {
            ent.push_back(pad);
            cnt[cur_d]++;
        }
        cur_d = -1;
    };
    int32_t cur_tile = -1;
    int64_t cur_src = -1, run_start_src = -1, run_pair0 = 0;
    bool pair_overflow = false;
    auto close_pair = [&]() {
        int64_t c = 0;
        for (int d = 0; d <= D; d++) {
            pair_doff.push_back((uint16_t)c);
            if (d < D) c += cnt[d];
        }
        pair_overflow |= c > 65535;
        std::fill(cnt.begin(), cnt.end(), 0);
    };
    auto close_run = [&]() {
        if (run_start_src >= 0)
            add_run(th, (uint32_t)run_start_src, (int32_t)(cur_src - run_start_src + 1), run_pair0, tile_D(cur_tile));
    };
    auto open_tiles_until = [&](int32_t q) {
        while ((int32_t)th.tile_units.size() <= q) {
            th.tile_units.push_back(0);
            const int32_t qq = (int32_t)th.tile_units.size() - 1;
            th.tile_run_off[qq + 1] = th.tile_run_off[qq];
        }
    };
    for (int64_t pos = 0; pos < s; pos++) {
        const int64_t k = key[pos].second;
        const int32_t q = (int32_t)(key[pos].first >> 37);
        if (q != cur_tile || src[k] != cur_src || delay[k] - 1 != cur_d) close_group();
        if (q != cur_tile || src[k] != cur_src) {
            if (cur_src >= 0) close_pair();
            const bool extends = q == cur_tile && src[k] == cur_src + 1;
            if (!extends) {
                if (cur_tile >= 0) close_run();
                open_tiles_until(q);
                run_start_src = src[k];
                run_pair0 = (int64_t)pair_base.size();
            }
            cur_tile = q;
            cur_src = src[k];
            pair_base.push_back((int64_t)ent.size());
        }
        cur_d = delay[k] - 1;
        cnt[cur_d]++;
        ent.push_back(make_uint2((uint32_t)(dst[k] - th.tile_beg[q]), f2u(weight[k])));
    }
    close_group();
    if (cur_src >= 0) {
        close_pair();
        close_run();
    }
    e.tile_entries.assign(nt, 0);
    for (int32_t q = 0; q < nt; q++)
        for (int32_t r = th.tile_run_off[q]; r < th.tile_run_off[q + 1]; r++)
            for (int32_t i = 0; i < th.run_n[r]; i++)
                e.tile_entries[q] += pair_doff[(size_t)(th.run_pair0[r] + i) * (D + 1) + D];
    open_tiles_until(nt - 1);
    if (pair_overflow) return fail(BSIM_ERR_LIMIT, "tiled delivery: a source has more than 65535 synapses into one tile");
    int64_t *d_pb;
    uint16_t *d_pd;
    uint2 *d_ent;
    TRY(dalloc(e, &d_pb, pair_base.size()));
    TRY(dalloc(e, &d_pd, pair_doff.size()));
    TRY(dalloc(e, &d_ent, ent.size()));
    if (!pair_base.empty()) {
        CK(cudaMemcpy(d_pb, pair_base.data(), 8 * pair_base.size(), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d_pd, pair_doff.data(), 2 * pair_doff.size(), cudaMemcpyHostToDevice));
    }
    if (!ent.empty()) CK(cudaMemcpy(d_ent, ent.data(), sizeof(uint2) * ent.size(), cudaMemcpyHostToDevice));
    e.a.pair_base = d_pb;
    e.a.pair_doff = d_pd;
    e.a.ent = d_ent;
    // pairs are grouped by tile: a tile's first pair is its first run's
    std::vector<int64_t> tile_pair0(nt + 1, (int64_t)pair_base.size());
    for (int32_t q = nt - 1; q >= 0; q--)
        tile_pair0[q] = th.tile_run_off[q] < th.tile_run_off[q + 1] ? th.run_pair0[th.tile_run_off[q]] : tile_pair0[q + 1];
    TRY(make_pair_seg(e, (int64_t)pair_base.size(), tile_pair0, th.tile_beg));
    return upload_tiles(e, th);
}

// ---------------------------------------------------------------------------
// Generated networks, built on the device.
// ---------------------------------------------------------------------------
#define GEN_MAX_DELAY 64
#define GEN_MAX_IN 8  // incoming projections per population handled by the device builder

struct GenInst {
    int64_t nbase;       // first global neuron id
    int32_t P, n, D;
    int32_t cls_base;    // class id of population 0 (class = cls_base + pop)
    uint64_t seed;
    uint32_t p24, exc24;
    float w_exc, w_inh;
    int32_t proj_off;    // into the projection table
    int32_t in_off;      // into the incoming table: [P][GEN_MAX_IN+1] (count, then projection ids)
    int32_t out_off;     // into the outgoing table: [P][3] (count, projection ids)
};

struct GenDev {
    const GenInst *inst;
    int32_t n_inst;
    const GenProj *proj;
    const int32_t *in_tab;
    const int32_t *out_tab;
    int32_t D;  // engine max delay
};

static __device__ __forceinline__ int find_inst(const GenDev &g, int64_t gid)
{
    int lo = 0, hi = g.n_inst - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (g.inst[mid].nbase <= gid) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Per-neuron state, v_tmp and class id. rm and Cm come from the host fold of
// each class so v_tmp = (i_offset*rm + v_rest) * (1 - Cm) rounds as on the host.
__global__ void gen_neurons_kernel(GenDev g, const bsim_gen_spec *specs, const float *cls_rm, const float *cls_Cm,
                                   float4 *state, float *vtmp, float *vtmp_alt, uint16_t *cls, int64_t N)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const int k = find_inst(g, i);
        const GenInst &gi = g.inst[k];
        const int64_t li = i - gi.nbase;
        const int pop = (int)(li / gi.n);
        const bsim_gen_spec &sp = specs[k];
        float ioff, vinit;
        draw_neuron(gi.seed, (uint64_t)li, sp, &ioff, &vinit);
        const int c = gi.cls_base + pop;
        const float rm = cls_rm[c], Cm = cls_Cm[c];
        float vt = __fadd_rn(__fmul_rn(ioff, rm), sp.v_rest);
        vt = __fmul_rn(vt, __fsub_rn(1.0f, Cm));
        vtmp[i] = vt;
        if (vtmp_alt) {
            // square-wave drive: the odd half periods' i_offset is i_offset * drive_scale
            const float ioff_hi = sp.drive_half_period > 0 ? __fmul_rn(ioff, sp.drive_scale) : ioff;
            float va = __fadd_rn(__fmul_rn(ioff_hi, rm), sp.v_rest);
            vtmp_alt[i] = __fmul_rn(va, __fsub_rn(1.0f, Cm));
        }
        cls[i] = (uint16_t)c;
        state[i] = make_float4(vinit, 0.0f, 0.0f, 0.0f);
    }
}

// Push rows: one warp per source neuron. Pass 0 counts entries per (source,
// delay); pass 1 writes them in creation order (projection, then target).
template <int PASS>
__global__ void gen_push_kernel(GenDev g, int64_t N, int64_t *row_cnt_or_off, uint2 *syn)
{
    __shared__ long long s_cur[8][GEN_MAX_DELAY];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int D = g.D;
    long long *cur = s_cur[wib];
    for (int64_t s = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < N;
         s += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int k = find_inst(g, s);
        const GenInst &gi = g.inst[k];
        const int64_t ls = s - gi.nbase;
        const int pop = (int)(ls / gi.n);
        const int64_t i = ls - (int64_t)pop * gi.n;
        for (int d = lane; d < D; d += 32) cur[d] = PASS == 0 ? 0 : row_cnt_or_off[s * D + d];
        __syncwarp();
        const int nout = g.out_tab[gi.out_off + 3 * pop];
        for (int q = 0; q < nout; q++) {
            const GenProj pr = g.proj[gi.proj_off + g.out_tab[gi.out_off + 3 * pop + 1 + q]];
            const int64_t tbase = gi.nbase + (int64_t)pr.dst_pop * gi.n;
            for (int j0 = 0; j0 < gi.n; j0 += 32) {
                const int j = j0 + lane;
                SynDraw sd;
                bool conn = j < gi.n && draw_pair(pr.pseed, (uint64_t)i, (uint64_t)j, gi.p24, gi.exc24, gi.w_exc,
                                                  gi.w_inh, gi.D, &sd);
                const unsigned m = __ballot_sync(0xffffffffu, conn);
                if (!m) continue;
                const unsigned same = __match_any_sync(0xffffffffu, conn ? sd.d : -1);
                if (conn) {
                    const int leader = __ffs(same) - 1;
                    const int rank = __popc(same & ((1u << lane) - 1u));
                    const long long at = cur[sd.d - 1] + rank;
                    if (PASS == 1) syn[at] = make_uint2((uint32_t)(tbase + j), __float_as_uint(sd.w));
                    __syncwarp(same);
                    if (lane == leader) cur[sd.d - 1] += __popc(same);
                }
                __syncwarp();
            }
        }
        __syncwarp();
        if (PASS == 0)
            for (int d = lane; d < D; d += 32) row_cnt_or_off[s * D + d] = cur[d];
        __syncwarp();
    }
}

// Pull rows: one warp per target neuron over its incoming projections in
// creation order, sources ascending inside a projection. Pass 0 counts and
// reduces the per-instance max in-degree and max |w|; pass 1 writes.
template <int PASS>
__global__ void gen_pull_kernel(GenDev g, int64_t N, int64_t *col_cnt_or_off, uint32_t *csrc, float *cw,
                                uint8_t *cd, unsigned long long *inst_maxdeg, unsigned int *inst_maxw)
{
    const int lane = threadIdx.x & 31;
    for (int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < N;
         t += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int k = find_inst(g, t);
        const GenInst &gi = g.inst[k];
        const int64_t lt = t - gi.nbase;
        const int pop = (int)(lt / gi.n);
        const int64_t j = lt - (int64_t)pop * gi.n;
        long long at = PASS == 0 ? 0 : col_cnt_or_off[t];
        float mw = 0.0f;
        const int nin = g.in_tab[gi.in_off + (GEN_MAX_IN + 1) * pop];
        for (int q = 0; q < nin; q++) {
            const GenProj pr = g.proj[gi.proj_off + g.in_tab[gi.in_off + (GEN_MAX_IN + 1) * pop + 1 + q]];
            const int64_t sbase = gi.nbase + (int64_t)pr.src_pop * gi.n;
            for (int i0 = 0; i0 < gi.n; i0 += 32) {
                const int i = i0 + lane;
                SynDraw sd;
                bool conn = i < gi.n && draw_pair(pr.pseed, (uint64_t)i, (uint64_t)j, gi.p24, gi.exc24, gi.w_exc,
                                                  gi.w_inh, gi.D, &sd);
                const unsigned m = __ballot_sync(0xffffffffu, conn);
                if (conn) {
                    const long long pos = at + __popc(m & ((1u << lane) - 1u));
                    if (PASS == 1) {
                        csrc[pos] = (uint32_t)(sbase + i);
                        cw[pos] = sd.w;
                        cd[pos] = (uint8_t)(sd.d - 1);
                    } else {
                        mw = fmaxf(mw, fabsf(sd.w));
                    }
                }
                at += __popc(m);
            }
        }
        if (PASS == 0) {
            for (int o = 16; o > 0; o >>= 1) mw = fmaxf(mw, __shfl_xor_sync(0xffffffffu, mw, o));
            if (lane == 0) {
                col_cnt_or_off[t] = at;
                atomicMax(&inst_maxdeg[k], (unsigned long long)at);
                atomicMax(&inst_maxw[k], __float_as_uint(mw));
            }
        }
    }
}

// One (tile, incoming projection) piece of the tiled copy: the sources of the
// projection's population against the targets [j0, j1) of its target
// population that lie in the tile. Its pairs are pair_start + source index.
struct TileSeg {
    int64_t pair_start;
    uint64_t pseed;
    int64_t src_base;   // global id of source 0
    int32_t j0, j1;     // target range, local to the target population
    int32_t tgt_off;    // offset of target j0 inside the tile
    int32_t n_src;
    uint32_t p24, exc24;
    float w_exc, w_inh;
    int32_t d_inst;     // the network's max delay
    int32_t sign;       // -1: all synapses; 0: excitatory only (w >= 0); 1: inhibitory only
};

static __device__ __forceinline__ int find_seg(const TileSeg *segs, int n_segs, int64_t k)
{
    int lo = 0, hi = n_segs - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (segs[mid].pair_start <= k) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// One warp per (tile, source) pair. Pass 0: per-delay counts -> cumulative
// pair_doff and pair_cnt (each delay's segment padded to even length). Pass 1:
// entries in delay order, targets ascending.
template <int PASS>
__global__ void gen_tile_kernel(const TileSeg *segs, int n_segs, int64_t n_pairs, int D,
                                int64_t *pair_cnt, uint16_t *pair_doff, const int64_t *pair_base,
                                uint2 *ent)
{
    __shared__ long long s_cur[8][GEN_MAX_DELAY];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    long long *cur = s_cur[wib];
    for (int64_t k = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < n_pairs;
         k += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const TileSeg sg = segs[find_seg(segs, n_segs, k)];
        const int64_t i = k - sg.pair_start;
        uint16_t *doff = pair_doff + k * (D + 1);
        for (int d = lane; d < D; d += 32) cur[d] = PASS == 0 ? 0 : pair_base[k] + doff[d];
        __syncwarp();
        for (int j0 = sg.j0; j0 < sg.j1; j0 += 32) {
            const int j = j0 + lane;
            SynDraw sd;
            bool conn = j < sg.j1 && draw_pair(sg.pseed, (uint64_t)i, (uint64_t)j, sg.p24, sg.exc24, sg.w_exc,
                                               sg.w_inh, sg.d_inst, &sd);
            if (conn && sg.sign >= 0) conn = (sd.w >= 0.0f) == (sg.sign == 0);
            if (!__ballot_sync(0xffffffffu, conn)) continue;
            const unsigned same = __match_any_sync(0xffffffffu, conn ? sd.d : -1);
            if (conn) {
                const int leader = __ffs(same) - 1;
                const long long at = cur[sd.d - 1] + __popc(same & ((1u << lane) - 1u));
                if (PASS == 1) ent[at] = make_uint2((uint32_t)(sg.tgt_off + (j - sg.j0)), __float_as_uint(sd.w));
                __syncwarp(same);
                if (lane == leader) cur[sd.d - 1] += __popc(same);
            }
            __syncwarp();
        }
        __syncwarp();
        if (PASS == 0 && lane == 0) {
            // segments padded to even length (the padding entries are preset)
            long long c = 0;
            for (int d = 0; d <= D; d++) {
                doff[d] = (uint16_t)c;
                if (d < D) c += (cur[d] + 1) & ~1ll;
            }
            pair_cnt[k] = c;
        }
        __syncwarp();
    }
}

static int check_spec(const bsim_gen_spec &g)
{
    if (g.n_pop < 1 || g.pop_size < 1 || g.max_delay < 1 || g.max_delay > GEN_MAX_DELAY ||
        (int64_t)g.n_pop * g.pop_size > (int64_t)INT32_MAX / 2 || !(g.p_conn >= 0) || g.p_conn > 1)
        return fail(BSIM_ERR_ARG, "bsim_gen_spec: invalid sizes (max_delay 1..64, p_conn in [0,1])");
    return BSIM_OK;
}

static int create_generated(const bsim_gen_spec *specs, int32_t ns, float dt, const bsim_options *opt, Engine **out)
{
    if (!specs || ns < 1 || !(dt > 0) || !out) return fail(BSIM_ERR_ARG, "bsim_create_generated: invalid arguments");
    std::vector<GenInst> gi(ns);
    std::vector<GenProj> proj;
    std::vector<int32_t> in_tab, out_tab;
    int64_t N = 0;
    int32_t D = 1, n_cls = 0;
    std::vector<ClassParams> ctab;
    std::vector<float> cls_rm, cls_Cm;
    std::vector<GenPlan> plans(ns);
    for (int k = 0; k < ns; k++) {
        const bsim_gen_spec &g = specs[k];
        TRY(check_spec(g));
        plans[k] = gen_plan(g);
        const GenPlan &pl = plans[k];
        GenInst &x = gi[k];
        x.nbase = N;
        x.P = g.n_pop;
        x.n = g.pop_size;
        x.D = g.max_delay;
        x.cls_base = n_cls;
        x.seed = g.seed;
        x.p24 = prob24(g.p_conn);
        x.exc24 = prob24(g.exc_frac);
        x.w_exc = g.w_max;
        x.w_inh = g.inh_scale * g.w_max;
        x.proj_off = (int32_t)proj.size();
        x.in_off = (int32_t)in_tab.size();
        x.out_off = (int32_t)out_tab.size();
        for (auto &p : pl.proj) proj.push_back(p);
        for (int p = 0; p < g.n_pop; p++) {
            if ((int)pl.in[p].size() > GEN_MAX_IN) return fail(BSIM_ERR_LIMIT, "generator: too many incoming projections");
            in_tab.push_back((int32_t)pl.in[p].size());
            for (int q = 0; q < GEN_MAX_IN; q++) in_tab.push_back(q < (int)pl.in[p].size() ? pl.in[p][q] : -1);
            out_tab.push_back((int32_t)pl.out[p].size());
            for (int q = 0; q < 2; q++) out_tab.push_back(q < (int)pl.out[p].size() ? pl.out[p][q] : -1);
        }
        N += (int64_t)g.n_pop * g.pop_size;
        D = std::max(D, g.max_delay);
        // one class per population; i_offset / v_init only change v_tmp and the initial state
        float prm[10];
        spec_params(g, 0.0f, 0.0f, prm);
        Folded f = fold_lif(prm, dt);
        const float ZERO = 1e-10f;
        float rm = fabsf(g.cm) > ZERO ? g.tau_m / g.cm : 1.0f;
        for (int p = 0; p < g.n_pop; p++) {
            ClassParams cp{};
            cp.Cm = f.Cm; cp.CE = f.CE; cp.CI = f.CI; cp.C_E = f.C_E; cp.C_I = f.C_I;
            cp.v_thresh = f.v_thresh; cp.v_reset = f.v_reset; cp.refrac_time = f.refrac_time;
            cp.pop = n_cls + p;
            cp.inst = k;
            cp.kind = BSIM_NEURON_LIF;
            cp.id_base = (int32_t)(N - (int64_t)g.n_pop * g.pop_size);
            ctab.push_back(cp);
            cls_rm.push_back(rm);
            cls_Cm.push_back(f.Cm);
        }
        n_cls += g.n_pop;
        if (n_cls > BSIM_MAX_CLASSES) return fail(BSIM_ERR_LIMIT, "generator: more than 65535 populations");
    }
    if (N > (int64_t)INT32_MAX - 64) return fail(BSIM_ERR_LIMIT, "generator: more than 2^31-64 neurons");

    Engine *e = new Engine();
    int rc = init_device(*e, opt);
    if (rc != BSIM_OK) { free_engine(e); return rc; }
    e->N = N;
    e->D = D;
    e->dt = dt;
    e->n_inst = ns;
    e->n_cls = n_cls;
    e->n_pops = n_cls;
    Engine &E = *e;
    auto bail = [&](int r) { free_engine(e); return r; };

    // small tables (freed at the end of the build)
    std::vector<void *> tmp;
    auto talloc = [&](void **p, size_t bytes) -> int {
        cudaError_t st = cudaMalloc(p, bytes ? bytes : 1);
        if (st != cudaSuccess) { cudaGetLastError(); return fail(BSIM_ERR_NOMEM, "build scratch allocation failed"); }
        tmp.push_back(*p);
        return BSIM_OK;
    };
    auto free_tmp = [&]() { for (void *p : tmp) cudaFree(p); tmp.clear(); };
    GenInst *d_gi; GenProj *d_proj; int32_t *d_in, *d_out; bsim_gen_spec *d_specs; float *d_rm, *d_Cm;
    if ((rc = talloc((void **)&d_gi, sizeof(GenInst) * ns)) || (rc = talloc((void **)&d_proj, sizeof(GenProj) * std::max<size_t>(1, proj.size()))) ||
        (rc = talloc((void **)&d_in, sizeof(int32_t) * in_tab.size())) || (rc = talloc((void **)&d_out, sizeof(int32_t) * out_tab.size())) ||
        (rc = talloc((void **)&d_specs, sizeof(bsim_gen_spec) * ns)) || (rc = talloc((void **)&d_rm, sizeof(float) * n_cls)) ||
        (rc = talloc((void **)&d_Cm, sizeof(float) * n_cls))) { free_tmp(); return bail(rc); }
    cudaMemcpy(d_gi, gi.data(), sizeof(GenInst) * ns, cudaMemcpyHostToDevice);
    if (!proj.empty()) cudaMemcpy(d_proj, proj.data(), sizeof(GenProj) * proj.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(d_in, in_tab.data(), sizeof(int32_t) * in_tab.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(d_out, out_tab.data(), sizeof(int32_t) * out_tab.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(d_specs, specs, sizeof(bsim_gen_spec) * ns, cudaMemcpyHostToDevice);
    cudaMemcpy(d_rm, cls_rm.data(), sizeof(float) * n_cls, cudaMemcpyHostToDevice);
    cudaMemcpy(d_Cm, cls_Cm.data(), sizeof(float) * n_cls, cudaMemcpyHostToDevice);
    GenDev gd{d_gi, ns, d_proj, d_in, d_out, D};

    int32_t drive_half = 0;
    for (int k = 0; k < ns; k++) {
        const int32_t h = specs[k].drive_half_period;
        if (h < 0 || (h > 0 && drive_half > 0 && h != drive_half)) {
            free_tmp();
            return bail(fail(BSIM_ERR_ARG, "generator: networks of one engine must share the drive half period"));
        }
        if (h > 0) drive_half = h;
    }
    float4 *d_state; float *d_vtmp, *d_vtmp_alt = nullptr; uint16_t *d_cls;
    if ((rc = dalloc(E, &d_state, N)) || (rc = dalloc(E, &d_vtmp, N)) || (rc = dalloc(E, &d_cls, N)) ||
        (drive_half > 0 && (rc = dalloc(E, &d_vtmp_alt, N)))) { free_tmp(); return bail(rc); }
    const int gb = E.sm_count * 8;
    gen_neurons_kernel<<<gb, 256, 0, E.stream>>>(gd, d_specs, d_rm, d_Cm, d_state, d_vtmp, d_vtmp_alt, d_cls, N);
    E.a.vtmp_alt = d_vtmp_alt;
    E.a.drive_half = drive_half;

    // in-degree and max |w| per instance -> fixed-point exponents
    int64_t *d_col;
    unsigned long long *d_maxdeg; unsigned int *d_maxw;
    if ((rc = dalloc(E, &d_col, N + 1)) || (rc = talloc((void **)&d_maxdeg, 8 * ns)) || (rc = talloc((void **)&d_maxw, 4 * ns))) { free_tmp(); return bail(rc); }
    cudaMemsetAsync(d_maxdeg, 0, 8 * ns, E.stream);
    cudaMemsetAsync(d_maxw, 0, 4 * ns, E.stream);
    cudaMemsetAsync(d_col + N, 0, 8, E.stream);
    gen_pull_kernel<0><<<gb, 256, 0, E.stream>>>(gd, N, d_col, nullptr, nullptr, nullptr, d_maxdeg, d_maxw);
    // exclusive scan of the counts (in place via a temp copy) -> col_off
    auto scan = [&](int64_t *arr, int64_t count) -> int {
        int64_t *d_tmp;
        if (talloc((void **)&d_tmp, sizeof(int64_t) * (count + 1))) return BSIM_ERR_NOMEM;
        cudaMemcpyAsync(d_tmp, arr, sizeof(int64_t) * count, cudaMemcpyDeviceToDevice, E.stream);
        cudaMemsetAsync(d_tmp + count, 0, 8, E.stream);
        size_t tb = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, tb, d_tmp, arr, count + 1, E.stream);
        void *d_tb;
        if (talloc(&d_tb, tb)) return BSIM_ERR_NOMEM;
        cub::DeviceScan::ExclusiveSum(d_tb, tb, d_tmp, arr, count + 1, E.stream);
        return BSIM_OK;
    };
    if ((rc = scan(d_col, N))) { free_tmp(); return bail(rc); }
    int64_t S = 0;
    std::vector<unsigned long long> maxdeg(ns);
    std::vector<unsigned int> maxw(ns);
    cudaMemcpyAsync(&S, d_col + N, 8, cudaMemcpyDeviceToHost, E.stream);
    cudaMemcpyAsync(maxdeg.data(), d_maxdeg, 8 * ns, cudaMemcpyDeviceToHost, E.stream);
    cudaMemcpyAsync(maxw.data(), d_maxw, 4 * ns, cudaMemcpyDeviceToHost, E.stream);
    if (cudaStreamSynchronize(E.stream) != cudaSuccess) { free_tmp(); return bail(fail(BSIM_ERR_CUDA, std::string("generator: ") + cudaGetErrorString(cudaGetLastError()))); }
    E.S = S;
    E.qexp.resize(ns);
    for (int k = 0; k < ns; k++) {
        float mw;
        memcpy(&mw, &maxw[k], 4);
        E.qexp[k] = choose_qexp((int64_t)maxdeg[k], mw);
    }
    for (auto &cp : ctab) {
        cp.scale_up = ldexpf(1.0f, E.qexp[cp.inst]);
        cp.scale_down = ldexpf(1.0f, -E.qexp[cp.inst]);
    }
    if (E.opt.build_pull) {
        uint32_t *d_csrc; float *d_cw; uint8_t *d_cd;
        if ((rc = dalloc(E, &d_csrc, S)) || (rc = dalloc(E, &d_cw, S)) || (rc = dalloc(E, &d_cd, S))) { free_tmp(); return bail(rc); }
        gen_pull_kernel<1><<<gb, 256, 0, E.stream>>>(gd, N, d_col, d_csrc, d_cw, d_cd, nullptr, nullptr);
        E.a.col_off = d_col;
        E.a.csc_src = d_csrc;
        E.a.csc_w = d_cw;
        E.a.csc_d = d_cd;
    }
    // target-tiled copy
    const bool tiles = wants_tiles(E.opt, D);
    if (tiles) {
        // target ranges follow population boundaries
        std::vector<int64_t> runs;
        for (int k = 0; k < ns; k++)
            for (int pp = 0; pp < gi[k].P; pp++) runs.push_back(gi[k].nbase + (int64_t)pp * gi[k].n);
        runs.push_back(N);
        std::vector<int32_t> tile_beg;
        int32_t tile_max = 0;
        plan_tiles(runs, auto_tile_size(E.opt, N, E.sm_count, D), tile_beg, tile_max);
        const int32_t nu = (int32_t)tile_beg.size() - 1, nt = nu;
        std::vector<TileSeg> segs;
        TileHost th;
        th.n_u = nu;
        th.tile_beg = tile_beg;
        th.tile_max = tile_max;
        th.tile_scale.resize(nt);
        th.tile_run_off.assign(nt + 1, 0);
        int64_t pairs = 0;
        std::vector<int64_t> tile_pair0(nt + 1, 0);
        for (int32_t q = 0; q < nt; q++) {
            const int32_t qu = q;
            tile_pair0[q] = pairs;
            int k = 0;
            while (k + 1 < ns && gi[k + 1].nbase <= tile_beg[qu]) k++;
            const GenInst &x = gi[k];
            const GenPlan &pl = plans[k];
            th.tile_units.push_back(0);
            th.tile_run_off[q + 1] = th.tile_run_off[q];
            th.tile_scale[q] = ldexpf(1.0f, E.qexp[k]);
            const int64_t lb = tile_beg[qu] - x.nbase, le = tile_beg[qu + 1] - x.nbase;
            for (int64_t pp = lb / x.n; pp <= (le - 1) / x.n; pp++) {
                const int64_t pop_beg = pp * x.n;
                const int32_t j0 = (int32_t)(std::max(lb, pop_beg) - pop_beg);
                const int32_t j1 = (int32_t)(std::min(le, pop_beg + x.n) - pop_beg);
                for (int id : pl.in[pp]) {
                    TileSeg sg;
                    sg.pair_start = pairs;
                    sg.pseed = pl.proj[id].pseed;
                    sg.src_base = x.nbase + (int64_t)pl.proj[id].src_pop * x.n;
                    sg.j0 = j0;
                    sg.j1 = j1;
                    sg.tgt_off = (int32_t)(pop_beg + j0 - lb);
                    sg.n_src = x.n;
                    sg.p24 = x.p24;
                    sg.exc24 = x.exc24;
                    sg.w_exc = x.w_exc;
                    sg.w_inh = x.w_inh;
                    sg.d_inst = x.D;
                    sg.sign = -1;
                    segs.push_back(sg);
                    add_run(th, (uint32_t)sg.src_base, x.n, pairs, x.D);  // the network's own delay range
                    pairs += x.n;
                }
            }
        }
        tile_pair0[nt] = pairs;
        TileSeg *d_segs;
        int64_t *d_pcnt;
        if ((rc = talloc((void **)&d_segs, sizeof(TileSeg) * std::max<size_t>(1, segs.size()))) ||
            (rc = talloc((void **)&d_pcnt, sizeof(int64_t) * (pairs + 1)))) { free_tmp(); return bail(rc); }
        if (!segs.empty()) cudaMemcpy(d_segs, segs.data(), sizeof(TileSeg) * segs.size(), cudaMemcpyHostToDevice);
        int64_t *d_pb; uint16_t *d_pd;
        if ((rc = dalloc(E, &d_pb, pairs + 1)) || (rc = dalloc(E, &d_pd, (size_t)pairs * (D + 1)))) {
            free_tmp();
            return bail(rc);
        }
        gen_tile_kernel<0><<<gb, 256, 0, E.stream>>>(d_segs, (int)segs.size(), pairs, D, d_pcnt, d_pd, nullptr,
                                                    nullptr);
        cudaMemcpyAsync(d_pb, d_pcnt, sizeof(int64_t) * pairs, cudaMemcpyDeviceToDevice, E.stream);
        if ((rc = scan(d_pb, pairs))) { free_tmp(); return bail(rc); }
        int64_t n_ent = 0;
        cudaMemcpyAsync(&n_ent, d_pb + pairs, 8, cudaMemcpyDeviceToHost, E.stream);
        if (cudaStreamSynchronize(E.stream) != cudaSuccess) {
            free_tmp();
            return bail(fail(BSIM_ERR_CUDA, "generator: tiled copy sizes"));
        }
        uint2 *d_ent;
        if ((rc = dalloc(E, &d_ent, n_ent))) { free_tmp(); return bail(rc); }
        cudaMemsetAsync(d_ent, 0xff, sizeof(uint2) * n_ent, E.stream);  // padding: target 0xffffffff
        gen_tile_kernel<1><<<gb, 256, 0, E.stream>>>(d_segs, (int)segs.size(), pairs, D, d_pcnt, d_pd, d_pb, d_ent);
        // entries per tile from the pair offsets at the tiles' first pairs
        std::vector<int64_t> pb_at(nt + 1, 0);
        for (int32_t q = 0; q <= nt; q++)
            cudaMemcpyAsync(&pb_at[q], d_pb + tile_pair0[q], 8, cudaMemcpyDeviceToHost, E.stream);
        if (cudaStreamSynchronize(E.stream) != cudaSuccess || pb_at[nt] != n_ent) {
            free_tmp();
            return bail(fail(BSIM_ERR_CUDA, "generator: tiled copy does not match its sizes"));
        }
        E.tile_entries.resize(nt);
        for (int32_t q = 0; q < nt; q++) E.tile_entries[q] = pb_at[q + 1] - pb_at[q];
        E.a.pair_base = d_pb;
        E.a.pair_doff = d_pd;
        E.a.ent = d_ent;
        if ((rc = make_pair_seg(E, pairs, tile_pair0, tile_beg))) { free_tmp(); return bail(rc); }
        if ((rc = upload_tiles(E, th))) { free_tmp(); return bail(rc); }
    }
    // push rows (not needed when every step uses the tiled copy)
    if (!(tiles && E.opt.delivery == BSIM_DELIVERY_TILE)) {
        const int64_t nrows = N * (int64_t)D;
        int64_t *d_row; uint2 *d_syn;
        if ((rc = dalloc(E, &d_row, nrows + 1)) || (rc = dalloc(E, &d_syn, S))) { free_tmp(); return bail(rc); }
        gen_push_kernel<0><<<gb, 256, 0, E.stream>>>(gd, N, d_row, nullptr);
        if ((rc = scan(d_row, nrows))) { free_tmp(); return bail(rc); }
        gen_push_kernel<1><<<gb, 256, 0, E.stream>>>(gd, N, d_row, d_syn);
        E.a.row_off = d_row;
        E.a.syn = d_syn;
    }
    cudaError_t st = cudaStreamSynchronize(E.stream);
    if (st == cudaSuccess) st = cudaGetLastError();
    free_tmp();
    if (st != cudaSuccess) return bail(fail(BSIM_ERR_CUDA, std::string("generator kernels: ") + cudaGetErrorString(st)));
    E.a.state = d_state;
    E.a.vtmp = d_vtmp;
    E.a.cls = d_cls;
    rc = finish_engine(E, ctab);
    if (rc != BSIM_OK) return bail(rc);
    *out = e;
    return BSIM_OK;
}

// Host generator: the same draws, emitted in global creation order (netgen.h).
static int gen_host(const bsim_gen_spec &g, float *params, int32_t *pop, int32_t *src, int32_t *dst, float *w,
                    int32_t *d, int64_t *n_out, int64_t *s_out)
{
    TRY(check_spec(g));
    netgen_host(g, params, pop, src, dst, w, d, n_out, s_out);
    return BSIM_OK;
}

}  // namespace bsim

using namespace bsim;

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
// The C handle is the engine itself behind an opaque pointer type.
static Engine *H(bsim_engine *h) { return reinterpret_cast<Engine *>(h); }
static bsim_engine *Hc(Engine *e) { return reinterpret_cast<bsim_engine *>(e); }

extern "C" {

int bsim_options_default(bsim_options *opt)
{
    if (!opt) return fail(BSIM_ERR_ARG, "null options");
    memset(opt, 0, sizeof(*opt));
    opt->device = 0;
    opt->accumulate = BSIM_ACC_EXACT;
    opt->delivery = BSIM_DELIVERY_PUSH;
    opt->build_pull = 0;
    opt->graph_steps = 64;
    return BSIM_OK;
}

int bsim_create(const float *params, int64_t n, const int32_t *pop, const int32_t *instance, const int32_t *src,
                const int32_t *dst, const float *weight, const int32_t *delay_steps, int64_t s, float dt,
                const bsim_options *opt, bsim_engine **out)
{
    Engine *e = nullptr;
    int rc = create_from_arrays(params, nullptr, n, pop, instance, src, dst, weight, delay_steps, s, dt, 0, opt, &e);
    if (rc == BSIM_OK) *out = Hc(e);
    return rc;
}

int bsim_create_mixed(const float *params, const uint8_t *kind, int64_t n, const int32_t *pop,
                      const int32_t *instance, const int32_t *src, const int32_t *dst, const float *weight,
                      const int32_t *delay_steps, int64_t s, float dt, uint64_t input_seed,
                      const bsim_options *opt, bsim_engine **out)
{
    Engine *e = nullptr;
    int rc = create_from_arrays(params, kind, n, pop, instance, src, dst, weight, delay_steps, s, dt, input_seed,
                                opt, &e);
    if (rc == BSIM_OK) *out = Hc(e);
    return rc;
}

int bsim_create_generated(const bsim_gen_spec *specs, int32_t n_specs, float dt, const bsim_options *opt,
                          bsim_engine **out)
{
    Engine *e = nullptr;
    int rc = create_generated(specs, n_specs, dt, opt, &e);
    if (rc == BSIM_OK) *out = Hc(e);
    return rc;
}

int bsim_gen_count(const bsim_gen_spec *spec, int64_t *n, int64_t *s)
{
    if (!spec) return fail(BSIM_ERR_ARG, "null spec");
    return gen_host(*spec, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, n, s);
}

int bsim_gen_host(const bsim_gen_spec *spec, float *params, int32_t *pop, int32_t *src, int32_t *dst, float *weight,
                  int32_t *delay_steps)
{
    if (!spec || !src || !dst || !weight || !delay_steps) return fail(BSIM_ERR_ARG, "null argument");
    return gen_host(*spec, params, pop, src, dst, weight, delay_steps, nullptr, nullptr);
}

int bsim_synapse_reset(const float *delay_s, const float *weight, const float *tau_syn, int64_t s, float dt,
                       int32_t *delay_steps, float *weight_out)
{
    if (s < 0 || (s > 0 && (!delay_s || !weight || !tau_syn || !delay_steps || !weight_out)))
        return fail(BSIM_ERR_ARG, "bsim_synapse_reset: invalid arguments");
    const float ZERO = 1e-10f;
    for (int64_t i = 0; i < s; i++) {
        int32_t st = (int32_t)roundf(delay_s[i] / dt);
        float rem = delay_s[i] - dt * (float)st;
        float w = weight[i];
        if (fabsf(tau_syn[i]) > ZERO && fabsf(rem) > ZERO) w = w * expf(-rem / tau_syn[i]);
        delay_steps[i] = st;
        weight_out[i] = w;
    }
    return BSIM_OK;
}

static int check_err(Engine &e)
{
    int32_t err = 0;
    CK(cudaMemcpy(&err, e.a.err, 4, cudaMemcpyDeviceToHost));
    if (err) {
        static const char *names[] = {"", "row offsets not ascending", "synapse target outside the network",
                                      "class index or kind out of range", "row offsets do not span the synapses",
                                      "a bounded wait inside the step ran out"};
        std::string m = "device error flag " + std::to_string(err);
        if (err > 0 && err <= 5) m += std::string(" (") + names[err] + ")";
        return fail(BSIM_ERR_DEVICE, m);
    }
    return BSIM_OK;
}

int bsim_run_async(bsim_engine *eh, int64_t steps)
{
    if (!eh || steps < 0) return fail(BSIM_ERR_ARG, "bsim_run: invalid arguments");
    Engine &e = *H(eh);
    CK(cudaSetDevice(e.device));
    int64_t left = steps;
    const int gl = e.opt.graph_steps;
    if (gl > 0 && left >= gl) {
        if (!e.graph_exec || e.graph_len != gl) {
            if (e.graph_exec) cudaGraphExecDestroy(e.graph_exec);
            if (e.graph) cudaGraphDestroy(e.graph);
            e.graph_exec = nullptr;
            e.graph = nullptr;
            CK(cudaStreamBeginCapture(e.stream, cudaStreamCaptureModeThreadLocal));
            for (int i = 0; i < gl; i++) {
                cudaError_t st = launch_step(e);
                if (st != cudaSuccess) {
                    cudaGraph_t g;
                    cudaStreamEndCapture(e.stream, &g);
                    if (g) cudaGraphDestroy(g);
                    return fail(BSIM_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(st));
                }
            }
            CK(cudaStreamEndCapture(e.stream, &e.graph));
            CK(cudaGraphInstantiate(&e.graph_exec, e.graph, 0));
            e.graph_len = gl;
        }
        while (left >= gl) {
            CK(cudaGraphLaunch(e.graph_exec, e.stream));
            left -= gl;
        }
    }
    for (; left > 0; left--) CK(launch_step(e));
    e.steps_done += steps;
    return BSIM_OK;
}

int bsim_sync(bsim_engine *eh)
{
    if (!eh) return fail(BSIM_ERR_ARG, "null engine");
    CK(cudaSetDevice(H(eh)->device));
    CK(cudaStreamSynchronize(H(eh)->stream));
    return check_err(*H(eh));
}

int bsim_stall_tile(bsim_engine *eh, int32_t tile)
{
    if (!eh) return fail(BSIM_ERR_ARG, "null engine");
    Engine &e = *H(eh);
    if (!e.a.tile_arrive || tile < 0 || tile >= e.a.n_tiles)
        return fail(BSIM_ERR_ARG, "bsim_stall_tile: the engine has no such tile");
    CK(cudaSetDevice(e.device));
    CK(cudaStreamSynchronize(e.stream));
    // the tile's finisher count of the running cycle (reset by the cycle's last block)
    const unsigned int one = 1u;
    CK(cudaMemcpy(e.a.tile_arrive + tile, &one, sizeof(one), cudaMemcpyHostToDevice));
    return BSIM_OK;
}

int bsim_run(bsim_engine *eh, int64_t steps)
{
    int rc = bsim_run_async(eh, steps);
    if (rc != BSIM_OK) return rc;
    return bsim_sync(eh);
}

// Scratch of the per-cycle sort of a recording of `items` ids over `segs` cycles.
static int sort_scratch_bytes(Engine &e, int64_t items, int64_t segs, size_t *bytes)
{
    *bytes = 0;
    CK(cub::DeviceSegmentedSort::SortKeys(nullptr, *bytes, e.a.rec_ids, e.rec_sorted, (int)std::max<int64_t>(items, 1),
                                          (int)std::max<int64_t>(segs, 1), e.a.rec_off, e.a.rec_off + 1, e.stream));
    return BSIM_OK;
}

int bsim_record(bsim_engine *eh, int64_t max_steps, int64_t capacity)
{
    if (!eh || max_steps < 0 || capacity < 0) return fail(BSIM_ERR_ARG, "bsim_record: invalid arguments");
    Engine &e = *H(eh);
    CK(cudaSetDevice(e.device));
    CK(cudaStreamSynchronize(e.stream));
    if (!e.a.rec) {
        RecCtl *rc;
        TRY(dalloc(e, &rc, 1));
        e.a.rec = rc;
        e.rec_dirty = true;
    }
    if (max_steps > e.rec_steps_alloc || capacity > e.rec_cap_alloc || !e.a.rec_ids) {
        // grow the buffers; the captured graph holds the old pointers
        int32_t *ids, *sorted;
        int64_t *off;
        const int64_t cap = std::max<int64_t>(capacity, e.rec_cap_alloc);
        const int64_t stp = std::max<int64_t>(max_steps, e.rec_steps_alloc);
        TRY(dalloc(e, &ids, cap));
        TRY(dalloc(e, &off, stp + 1));
        e.a.rec_ids = ids;
        e.a.rec_off = off;
        e.rec_cap_alloc = cap;
        e.rec_steps_alloc = stp;
        e.rec_dirty = true;
        // the read-back's sorted copy and sort scratch, sized for a full recording
        // (recordings of 2^31 ids or more are sorted on the host and need neither)
        e.rec_sorted = nullptr;  // the old sorted copy is too small for the new buffers
        if (cap < ((int64_t)1 << 31) && stp < ((int64_t)1 << 31)) {
            TRY(dalloc(e, &sorted, cap));
            e.rec_sorted = sorted;
            size_t tb = 0;
            TRY(sort_scratch_bytes(e, cap, stp, &tb));
            if (tb > e.sort_tmp_bytes) {
                char *tmp;
                TRY(dalloc(e, &tmp, tb));
                e.sort_tmp = tmp;
                e.sort_tmp_bytes = tb;
            }
        }
    }
    RecCtl ctl{e.steps_done, e.steps_done, max_steps, capacity};
    CK(cudaMemset(e.a.rec_off, 0, sizeof(int64_t)));
    CK(cudaMemcpy(e.a.rec, &ctl, sizeof(ctl), cudaMemcpyHostToDevice));
    if (e.rec_dirty) {
        if (e.graph_exec) { cudaGraphExecDestroy(e.graph_exec); e.graph_exec = nullptr; }
        if (e.graph) { cudaGraphDestroy(e.graph); e.graph = nullptr; }
        e.rec_dirty = false;
    }
    return BSIM_OK;
}

int bsim_read_raster(bsim_engine *eh, int64_t *step_off, int32_t *ids, int64_t ids_cap, int64_t *n_steps)
{
    if (!eh || !step_off || !n_steps) return fail(BSIM_ERR_ARG, "bsim_read_raster: invalid arguments");
    Engine &e = *H(eh);
    if (!e.a.rec || !e.a.rec_ids) return fail(BSIM_ERR_STATE, "bsim_read_raster: recording not enabled");
    CK(cudaSetDevice(e.device));
    CK(launch_record_flush(e));
    RecCtl ctl;
    CK(cudaMemcpyAsync(&ctl, e.a.rec, sizeof(ctl), cudaMemcpyDeviceToHost, e.stream));
    CK(cudaStreamSynchronize(e.stream));
    int64_t ns = ctl.next - ctl.t0;
    if (ns < 0) ns = 0;
    if (ns > ctl.steps) ns = ctl.steps;
    CK(cudaMemcpy(step_off, e.a.rec_off, sizeof(int64_t) * (ns + 1), cudaMemcpyDeviceToHost));
    *n_steps = ns;
    int64_t total = step_off[ns];
    if (total > ctl.cap) return fail(BSIM_ERR_LIMIT, "raster buffer overflowed");
    if (ids) {
        if (total > ids_cap) return fail(BSIM_ERR_ARG, "bsim_read_raster: ids buffer too small");
        if (total == 0) return BSIM_OK;
        // ascending ids within each cycle: one segmented sort on the device (the
        // cycles' segments tile the recording) into the buffers bsim_record set up;
        // recordings of 2^31 ids or more are sorted on the host
        if (!e.rec_sorted || total >= ((int64_t)1 << 31) || ns >= ((int64_t)1 << 31)) {
            CK(cudaMemcpy(ids, e.a.rec_ids, sizeof(int32_t) * total, cudaMemcpyDeviceToHost));
            for (int64_t k = 0; k < ns; k++) std::sort(ids + step_off[k], ids + step_off[k + 1]);
            return BSIM_OK;
        }
        size_t tmp_bytes = 0;
        TRY(sort_scratch_bytes(e, total, ns, &tmp_bytes));
        if (tmp_bytes > e.sort_tmp_bytes) {  // not expected: the scratch was sized for a full recording
            char *tmp;
            TRY(dalloc(e, &tmp, tmp_bytes));
            e.sort_tmp = tmp;
            e.sort_tmp_bytes = tmp_bytes;
        }
        size_t tb = e.sort_tmp_bytes;
        CK(cub::DeviceSegmentedSort::SortKeys(e.sort_tmp, tb, e.a.rec_ids, e.rec_sorted, (int)total, (int)ns,
                                              e.a.rec_off, e.a.rec_off + 1, e.stream));
        CK(cudaMemcpyAsync(ids, e.rec_sorted, sizeof(int32_t) * total, cudaMemcpyDeviceToHost, e.stream));
        CK(cudaStreamSynchronize(e.stream));
    }
    return BSIM_OK;
}

int bsim_trace(bsim_engine *eh, int64_t max_steps, int64_t first, int64_t count)
{
    if (!eh || max_steps < 0 || first < 0 || count < 0) return fail(BSIM_ERR_ARG, "bsim_trace: invalid arguments");
    Engine &e = *H(eh);
    if (first + count > e.N) return fail(BSIM_ERR_ARG, "bsim_trace: neuron range beyond the network");
    CK(cudaSetDevice(e.device));
    CK(cudaStreamSynchronize(e.stream));
    bool dirty = false;
    if (!e.a.trace_ctl) {
        TraceCtl *tc;
        TRY(dalloc(e, &tc, 1));
        e.a.trace_ctl = tc;
        dirty = true;
    }
    const int64_t need = 5 * max_steps * count;
    if (need > e.trace_alloc || !e.a.trace) {
        float *buf;
        TRY(dalloc(e, &buf, std::max<int64_t>(need, 1)));
        e.a.trace = buf;
        e.trace_alloc = std::max<int64_t>(need, 1);
        dirty = true;
    }
    TraceCtl ctl{e.steps_done, max_steps, first, count};
    CK(cudaMemcpy(const_cast<TraceCtl *>(e.a.trace_ctl), &ctl, sizeof(ctl), cudaMemcpyHostToDevice));
    if (dirty) {  // the captured graph holds the old arguments
        if (e.graph_exec) { cudaGraphExecDestroy(e.graph_exec); e.graph_exec = nullptr; }
        if (e.graph) { cudaGraphDestroy(e.graph); e.graph = nullptr; }
    }
    return BSIM_OK;
}

int bsim_read_trace(bsim_engine *eh, float *v, float *iE, float *iI, float *in_E, float *in_I, int64_t *n_steps)
{
    if (!eh || !n_steps) return fail(BSIM_ERR_ARG, "bsim_read_trace: invalid arguments");
    Engine &e = *H(eh);
    if (!e.a.trace || !e.a.trace_ctl) return fail(BSIM_ERR_STATE, "bsim_read_trace: tracing not enabled");
    CK(cudaSetDevice(e.device));
    TraceCtl ctl;
    CK(cudaMemcpyAsync(&ctl, e.a.trace_ctl, sizeof(ctl), cudaMemcpyDeviceToHost, e.stream));
    unsigned long long done = 0;
    CK(cudaMemcpyAsync(&done, e.a.step_ctr, sizeof(done), cudaMemcpyDeviceToHost, e.stream));
    CK(cudaStreamSynchronize(e.stream));
    int64_t ns = (int64_t)done - ctl.t0;
    ns = std::max<int64_t>(0, std::min<int64_t>(ns, ctl.steps));
    *n_steps = ns;
    float *dst[5] = {v, iE, iI, in_E, in_I};
    const int64_t plane = ctl.steps * ctl.count;
    for (int f = 0; f < 5; f++)
        if (dst[f] && ns > 0)
            CK(cudaMemcpyAsync(dst[f], e.a.trace + f * plane, sizeof(float) * ns * ctl.count, cudaMemcpyDeviceToHost,
                               e.stream));
    CK(cudaStreamSynchronize(e.stream));
    return BSIM_OK;
}

// The state's four fields as planes of N words in the staging buffer (read-back),
// and back (upload; a NULL plane leaves its field).
__global__ void state_unpack_kernel(const float4 *st, float *stage, int64_t n)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float4 s = st[i];
        stage[i] = s.x;
        stage[n + i] = s.y;
        stage[2 * n + i] = s.z;
        stage[3 * n + i] = s.w;
    }
}

__global__ void state_pack_kernel(float4 *st, const float *stage, int64_t n, int has_v, int has_ie, int has_ii,
                                  int has_rf)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float4 s = st[i];
        if (has_v) s.x = stage[i];
        if (has_ie) s.y = stage[n + i];
        if (has_ii) s.z = stage[2 * n + i];
        if (has_rf) s.w = stage[3 * n + i];
        st[i] = s;
    }
}

static int ensure_stage(Engine &e)
{
    if (e.stage) return BSIM_OK;
    float *d;
    TRY(dalloc(e, &d, 4 * (size_t)e.N));
    e.stage = d;
    return BSIM_OK;
}

static int state_grid(const Engine &e) { return (int)std::min<int64_t>((e.N + 255) / 256, 8 * (int64_t)e.sm_count); }

int bsim_read_state(bsim_engine *eh, float *v, float *iE, float *iI, int32_t *refrac)
{
    if (!eh) return fail(BSIM_ERR_ARG, "null engine");
    Engine &e = *H(eh);
    CK(cudaSetDevice(e.device));
    TRY(ensure_stage(e));
    state_unpack_kernel<<<state_grid(e), 256, 0, e.stream>>>(e.a.state, e.stage, e.N);
    CK(cudaGetLastError());
    void *dst[4] = {v, iE, iI, refrac};
    for (int k = 0; k < 4; k++)
        if (dst[k])
            CK(cudaMemcpyAsync(dst[k], e.stage + (size_t)k * e.N, sizeof(float) * e.N, cudaMemcpyDeviceToHost,
                               e.stream));
    CK(cudaStreamSynchronize(e.stream));
    return BSIM_OK;
}

int bsim_write_state(bsim_engine *eh, const float *v, const float *iE, const float *iI, const int32_t *refrac)
{
    if (!eh) return fail(BSIM_ERR_ARG, "null engine");
    Engine &e = *H(eh);
    CK(cudaSetDevice(e.device));
    TRY(ensure_stage(e));
    const void *src[4] = {v, iE, iI, refrac};
    for (int k = 0; k < 4; k++)
        if (src[k])
            CK(cudaMemcpyAsync(e.stage + (size_t)k * e.N, src[k], sizeof(float) * e.N, cudaMemcpyHostToDevice,
                               e.stream));
    state_pack_kernel<<<state_grid(e), 256, 0, e.stream>>>(e.a.state, e.stage, e.N, v != nullptr, iE != nullptr,
                                                            iI != nullptr, refrac != nullptr);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(e.stream));
    return BSIM_OK;
}

int bsim_set_drive(bsim_engine *eh, const float *params_hi, int32_t half_period)
{
    if (!eh || half_period < 0 || (half_period > 0 && !params_hi)) return fail(BSIM_ERR_ARG, "bsim_set_drive: invalid arguments");
    Engine &e = *H(eh);
    CK(cudaSetDevice(e.device));
    CK(cudaStreamSynchronize(e.stream));
    if (half_period > 0) {
        std::vector<float> vt(e.N);
        const float dt = e.dt;
        for (int64_t i = 0; i < e.N; i++) vt[i] = fold_lif(params_hi + 10 * i, dt).v_tmp;
        if (!e.a.vtmp_alt) {
            float *d;
            TRY(dalloc(e, &d, e.N));
            e.a.vtmp_alt = d;
        }
        CK(cudaMemcpy(const_cast<float *>(e.a.vtmp_alt), vt.data(), sizeof(float) * e.N, cudaMemcpyHostToDevice));
    }
    e.a.drive_half = half_period;
    // the captured graph holds the old arguments
    if (e.graph_exec) { cudaGraphExecDestroy(e.graph_exec); e.graph_exec = nullptr; }
    if (e.graph) { cudaGraphDestroy(e.graph); e.graph = nullptr; }
    return BSIM_OK;
}

int bsim_get_stream(bsim_engine *eh, void **stream)
{
    if (!eh || !stream) return fail(BSIM_ERR_ARG, "invalid arguments");
    *stream = (void *)H(eh)->stream;
    return BSIM_OK;
}

int bsim_read_fire_count(bsim_engine *eh, int32_t *count)
{
    if (!eh || !count) return fail(BSIM_ERR_ARG, "invalid arguments");
    Engine &e = *H(eh);
    CK(cudaSetDevice(e.device));
    CK(cudaMemcpyAsync(count, e.a.fire_count, sizeof(int32_t) * e.N, cudaMemcpyDeviceToHost, e.stream));
    CK(cudaStreamSynchronize(e.stream));
    return BSIM_OK;
}

static void drop_graph(Engine &e)
{
    if (e.graph_exec) { cudaGraphExecDestroy(e.graph_exec); e.graph_exec = nullptr; }
    if (e.graph) { cudaGraphDestroy(e.graph); e.graph = nullptr; }
}

// Per-population size and summed in/out degree, from whichever copies of the
// synapses the engine holds (push rows, pull rows or the tiled copy).
__global__ void pop_degree_kernel(StepArgs a, int32_t *size, double *in_sum, double *out_sum)
{
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < a.N; j += (int64_t)gridDim.x * blockDim.x) {
        const int pop = a.ctab[a.cls[j]].pop;
        atomicAdd(&size[pop], 1);
        if (a.col_off) atomicAdd(&in_sum[pop], (double)(a.col_off[j + 1] - a.col_off[j]));
        if (a.row_off) atomicAdd(&out_sum[pop], (double)(a.row_off[(j + 1) * a.D] - a.row_off[j * a.D]));
    }
}

// In-degree of every neuron from the push rows (when no target-ordered copy exists).
__global__ void indeg_from_push_kernel(StepArgs a, int32_t *indeg)
{
    const int64_t S = a.row_off[a.N * a.D];
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < S; k += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(&indeg[a.syn[k].x], 1);
}

__global__ void pop_in_from_counts_kernel(StepArgs a, const int32_t *indeg, double *in_sum)
{
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < a.N; j += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(&in_sum[a.ctab[a.cls[j]].pop], (double)indeg[j]);
}

__global__ void pop_degree_tiles_kernel(StepArgs a, double *in_sum, double *out_sum, int want_in, int want_out)
{
    // one block per tile: entries per pair give out-degree of the source and in-degree of the tile
    for (int q = blockIdx.x; q < a.n_tiles; q += gridDim.x) {
        for (int r = a.tile_run_off[q]; r < a.tile_run_off[q + 1]; r++) {
            for (int i = threadIdx.x; i < a.run_n[r]; i += blockDim.x) {
                const int64_t k = a.run_pair0[r] + i;
                const int64_t b = a.pair_base[k], n_e = a.pair_doff[k * (a.D + 1) + a.D];
                int64_t real = 0;
                for (int64_t x = 0; x < n_e; x++) real += a.ent[b + x].x != TILE_PAD;
                const double c = (double)real;
                const uint32_t src = a.run_src0[r] + i;
                if (want_out) atomicAdd(&out_sum[a.ctab[a.cls[src]].pop], c);
                if (want_in) atomicAdd(&in_sum[a.ctab[a.cls[a.tile_beg[q]]].pop], c);
            }
        }
    }
}

static int ensure_pop_info(Engine &e)
{
    if (e.pop_info_ready) return BSIM_OK;
    const int P = e.n_pops;
    int32_t *d_size;
    double *d_in, *d_out;
    float *d_ind, *d_outd;
    TRY(dalloc(e, &d_size, P));
    TRY(dalloc(e, &d_in, P));
    TRY(dalloc(e, &d_out, P));
    TRY(dalloc(e, &d_ind, P));
    TRY(dalloc(e, &d_outd, P));
    CK(cudaMemset(d_size, 0, 4 * P));
    CK(cudaMemset(d_in, 0, 8 * P));
    CK(cudaMemset(d_out, 0, 8 * P));
    pop_degree_kernel<<<e.sm_count * 4, 256, 0, e.stream>>>(e.a, d_size, d_in, d_out);
    bool in_done = e.a.col_off != nullptr;
    if (!in_done && e.a.row_off) {
        int32_t *d_indeg = nullptr;
        CK(cudaMalloc((void **)&d_indeg, sizeof(int32_t) * e.N));
        cudaMemsetAsync(d_indeg, 0, sizeof(int32_t) * e.N, e.stream);
        indeg_from_push_kernel<<<e.sm_count * 8, 256, 0, e.stream>>>(e.a, d_indeg);
        pop_in_from_counts_kernel<<<e.sm_count * 4, 256, 0, e.stream>>>(e.a, d_indeg, d_in);
        cudaError_t st = cudaStreamSynchronize(e.stream);
        cudaFree(d_indeg);
        if (st != cudaSuccess) return fail(BSIM_ERR_CUDA, std::string("population degrees: ") + cudaGetErrorString(st));
        in_done = true;
    }
    if (e.a.n_tiles > 0 && (!in_done || !e.a.row_off))
        pop_degree_tiles_kernel<<<e.sm_count * 4, 256, 0, e.stream>>>(e.a, d_in, d_out, in_done ? 0 : 1,
                                                                      e.a.row_off ? 0 : 1);
    CK(cudaStreamSynchronize(e.stream));
    std::vector<int32_t> sz(P);
    std::vector<double> in(P), out(P);
    std::vector<float> ind(P), outd(P);
    CK(cudaMemcpy(sz.data(), d_size, 4 * P, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(in.data(), d_in, 8 * P, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(out.data(), d_out, 8 * P, cudaMemcpyDeviceToHost));
    for (int p = 0; p < P; p++) {
        ind[p] = sz[p] ? (float)(in[p] / sz[p]) : 0.0f;
        outd[p] = sz[p] ? (float)(out[p] / sz[p]) : 0.0f;
    }
    CK(cudaMemcpy(d_ind, ind.data(), 4 * P, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_outd, outd.data(), 4 * P, cudaMemcpyHostToDevice));
    e.a.pop_size = d_size;
    e.a.pop_indeg = d_ind;
    e.a.pop_outdeg = d_outd;
    e.pop_info_ready = true;
    return BSIM_OK;
}

int bsim_enable_pop_stats(bsim_engine *eh, int32_t hist_len)
{
    if (!eh || hist_len < 16) return fail(BSIM_ERR_ARG, "bsim_enable_pop_stats: hist_len must be >= 16");
    Engine &e = *H(eh);
    CK(cudaSetDevice(e.device));
    CK(cudaStreamSynchronize(e.stream));
    TRY(ensure_pop_info(e));
    if (e.a.pop_hist && e.a.hist_len == hist_len) return BSIM_OK;
    int32_t *h;
    TRY(dalloc(e, &h, (size_t)hist_len * e.n_pops));
    CK(cudaMemset(h, 0, sizeof(int32_t) * hist_len * e.n_pops));
    e.a.pop_hist = h;
    e.a.hist_len = hist_len;
    drop_graph(e);
    return BSIM_OK;
}

int bsim_read_pop_counts(bsim_engine *eh, int32_t *counts, int32_t steps)
{
    if (!eh || !counts || steps < 0) return fail(BSIM_ERR_ARG, "bsim_read_pop_counts: invalid arguments");
    Engine &e = *H(eh);
    if (!e.a.pop_hist) return fail(BSIM_ERR_STATE, "population statistics are not enabled on this engine");
    if (steps > e.a.hist_len - 2) return fail(BSIM_ERR_ARG, "bsim_read_pop_counts: steps > hist_len - 2");
    CK(cudaSetDevice(e.device));
    CK(cudaStreamSynchronize(e.stream));
    const int H = e.a.hist_len, P = e.n_pops;
    std::vector<int32_t> ring((size_t)H * P);
    CK(cudaMemcpy(ring.data(), e.a.pop_hist, sizeof(int32_t) * H * P, cudaMemcpyDeviceToHost));
    const int64_t T = e.steps_done;
    for (int32_t k = 0; k < steps; k++) {
        const int64_t s = T - steps + k;
        for (int p = 0; p < P; p++) counts[(int64_t)k * P + p] = s >= 0 ? ring[(size_t)(s % H) * P + p] : 0;
    }
    return BSIM_OK;
}

int bsim_read_pop_info(bsim_engine *eh, int32_t *size, float *mean_indeg, float *mean_outdeg)
{
    if (!eh) return fail(BSIM_ERR_ARG, "null engine");
    Engine &e = *H(eh);
    CK(cudaSetDevice(e.device));
    CK(cudaStreamSynchronize(e.stream));
    TRY(ensure_pop_info(e));
    const int P = e.n_pops;
    if (size) CK(cudaMemcpy(size, e.a.pop_size, 4 * P, cudaMemcpyDeviceToHost));
    if (mean_indeg) CK(cudaMemcpy(mean_indeg, e.a.pop_indeg, 4 * P, cudaMemcpyDeviceToHost));
    if (mean_outdeg) CK(cudaMemcpy(mean_outdeg, e.a.pop_outdeg, 4 * P, cudaMemcpyDeviceToHost));
    return BSIM_OK;
}

int bsim_set_predictor(bsim_engine *eh, const float *params, float tolerance, const float *cost_push,
                       const float *cost_tile)
{
    if (!eh || (params && !(tolerance >= 0))) return fail(BSIM_ERR_ARG, "bsim_set_predictor: invalid arguments");
    Engine &e = *H(eh);
    CK(cudaSetDevice(e.device));
    CK(cudaStreamSynchronize(e.stream));
    if (!params && !cost_push && !cost_tile) {  // detached: AUTO pushes every cycle
        e.a.mlp = nullptr;
        e.a.pstats = nullptr;
        drop_graph(e);
        return BSIM_OK;
    }
    if (params && !e.a.pop_hist) return fail(BSIM_ERR_STATE, "bsim_set_predictor: enable population statistics first");
    if (!e.pstats_mem) {
        PredStats *ps;
        TRY(dalloc(e, &ps, 1));
        e.pstats_mem = ps;
    }
    e.a.pstats = e.pstats_mem;
    CK(cudaMemset(e.a.pstats, 0, sizeof(PredStats)));
    if (!params) {  // the exact schedule: the cost models on the delivered window's spike count
        e.a.mlp = nullptr;
    } else {
        if (!e.mlp_mem) {
            float *w, *ring, *sum;
            TRY(dalloc(e, &w, BSIM_MLP_PARAMS));
            TRY(dalloc(e, &ring, 4 * (size_t)e.n_pops));
            TRY(dalloc(e, &sum, 8));
            e.mlp_mem = w;
            e.a.pred_ring = ring;
            e.a.pred_sum = sum;
        }
        e.a.mlp = e.mlp_mem;
        CK(cudaMemcpy(e.mlp_mem, params, sizeof(float) * BSIM_MLP_PARAMS, cudaMemcpyHostToDevice));
        CK(cudaMemset(e.a.pred_ring, 0, sizeof(float) * 4 * e.n_pops));
        CK(cudaMemset(e.a.pred_sum, 0, sizeof(float) * 8));
    }
    e.a.pred_tol = tolerance;
    e.a.mean_outdeg = e.N ? (float)((double)e.S / (double)e.N) : 0.0f;
    e.a.cost_push_a = cost_push ? cost_push[0] : 0.0f;
    e.a.cost_push_b = cost_push ? cost_push[1] : 1.0f;
    e.a.cost_tile_a = cost_tile ? cost_tile[0] : 0.0f;
    e.a.cost_tile_b = cost_tile ? cost_tile[1] : 2.0f;
    drop_graph(e);
    return BSIM_OK;
}

int bsim_predictor_stats(bsim_engine *eh, bsim_pred_stats *st)
{
    if (!eh || !st) return fail(BSIM_ERR_ARG, "invalid arguments");
    Engine &e = *H(eh);
    memset(st, 0, sizeof(*st));
    if (!e.a.pstats) return BSIM_OK;
    CK(cudaSetDevice(e.device));
    CK(cudaStreamSynchronize(e.stream));
    PredStats ps;
    CK(cudaMemcpy(&ps, e.a.pstats, sizeof(ps), cudaMemcpyDeviceToHost));
    st->cycles = (int64_t)ps.cycles;
    st->fallbacks = (int64_t)ps.fallbacks;
    st->tile_cycles = (int64_t)ps.tile_cycles;
    st->abs_err_sum = ps.abs_err;
    st->actual_sum = ps.actual;
    return BSIM_OK;
}

int bsim_autotune(bsim_engine *eh, int32_t trial_steps, bsim_tune_result *out)
{
    if (!eh || trial_steps < 1 || !out) return fail(BSIM_ERR_ARG, "bsim_autotune: invalid arguments");
    Engine &e = *H(eh);
    CK(cudaSetDevice(e.device));
    CK(cudaStreamSynchronize(e.stream));
    memset(out, 0, sizeof(*out));
    if (e.opt.accumulate == BSIM_ACC_ORDERED) {  // one schedule only
        out->block_threads = e.block;
        out->grid_blocks = e.grid;
        out->delivery = BSIM_DELIVERY_PULL;
        return BSIM_OK;
    }
    if (!e.a.acc_clear) {
        // The trials switch modes, and push adds into the planes: from here on the
        // LIF phase clears them. The parity the next cycle delivers into holds the
        // input consumed by the last cycle; zero it (the other parity is unread input).
        unsigned long long t_next = 0;
        CK(cudaMemcpy(&t_next, e.a.step_ctr, sizeof(t_next), cudaMemcpyDeviceToHost));
        const size_t plane_set = (size_t)e.a.n_planes * (size_t)e.N;
        CK(cudaMemset(reinterpret_cast<longlong2 *>(e.a.acc) + ((t_next & 1ull) ^ 1ull) * plane_set, 0,
                      sizeof(longlong2) * plane_set));
        e.a.acc_clear = 1;
        drop_graph(e);
    }
    std::vector<int> modes;
    if (e.a.row_off) modes.push_back(BSIM_DELIVERY_PUSH);
    if (e.a.n_tiles > 0) modes.push_back(BSIM_DELIVERY_TILE);
    const int saved_block = e.block, saved_grid = e.grid, saved_del = e.a.delivery;
    cudaEvent_t ev0, ev1;
    CK(cudaEventCreate(&ev0));
    CK(cudaEventCreate(&ev1));
    // Candidates: delivery mode x block size x grid. The network's activity drifts
    // while the trials run (they advance the simulation), so the candidates take
    // turns over several rounds and are compared on their summed time.
    struct Cand { int m, b, g; float ms; unsigned long long ev; };
    std::vector<Cand> cands;
    const int blocks[2] = {256, 512};
    for (int m : modes)
        for (int b : blocks) {
            int bps = 0;
            const size_t smem = step_dynamic_smem(e.a, b);
            if (smem > 0) CK(step_set_smem(e.opt.accumulate, smem));
            if (step_occupancy(b, e.opt.accumulate, &bps, smem) != cudaSuccess || bps < 1) continue;
            const int grids[2] = {e.sm_count * bps, e.sm_count};
            for (int g : grids) cands.push_back(Cand{m, b, g, 0.0f, 0ull});
        }
    const int rounds = 3;
    for (int r = 0; r < rounds; r++) {
        for (Cand &c : cands) {
            e.block = c.b;
            e.grid = c.g;
            e.a.delivery = c.m;
            unsigned long long c0[2], c1[2];
            CK(cudaMemcpy(c0, e.a.step_ctr, sizeof(c0), cudaMemcpyDeviceToHost));
            CK(cudaEventRecord(ev0, e.stream));
            for (int k = 0; k < trial_steps; k++) CK(launch_step(e));
            CK(cudaEventRecord(ev1, e.stream));
            CK(cudaEventSynchronize(ev1));
            float ms = 0.0f;
            CK(cudaEventElapsedTime(&ms, ev0, ev1));
            CK(cudaMemcpy(c1, e.a.step_ctr, sizeof(c1), cudaMemcpyDeviceToHost));
            e.steps_done += trial_steps;
            c.ms += ms;
            c.ev += c1[1] - c0[1];
        }
    }
    out->candidates = (int32_t)cands.size();
    float best = 1e30f;
    int best_b = saved_block, best_g = saved_grid, best_m = saved_del;
    float mode_best[4] = {1e30f, 1e30f, 1e30f, 1e30f};
    unsigned long long mode_ev[4] = {0, 0, 0, 0};
    for (const Cand &c : cands) {
        const float us = 1e3f * c.ms / (float)(rounds * trial_steps);
        if (us < best) {
            best = us;
            best_b = c.b;
            best_g = c.g;
            best_m = c.m;
        }
        if (us < mode_best[c.m]) {
            mode_best[c.m] = us;
            mode_ev[c.m] = c.ev / (unsigned long long)(rounds * trial_steps);
        }
    }
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    e.block = best_b;
    e.grid = best_g;
    // an AUTO engine keeps choosing per cycle; a fixed one takes the fastest mode
    if (saved_del == BSIM_DELIVERY_AUTO) {
        e.a.delivery = BSIM_DELIVERY_AUTO;
    } else {
        e.a.delivery = best_m;
        e.opt.delivery = best_m;
    }
    drop_graph(e);
    out->block_threads = best_b;
    out->grid_blocks = best_g;
    out->delivery = best_m;
    out->best_us_per_step = best;
    // cost model of each mode: ns per event at the trial's activity (fixed part not separated)
    if (mode_best[BSIM_DELIVERY_PUSH] < 1e29f && mode_ev[BSIM_DELIVERY_PUSH] > 0)
        out->cost_push[1] = 1e3f * mode_best[BSIM_DELIVERY_PUSH] / (float)mode_ev[BSIM_DELIVERY_PUSH];
    if (mode_best[BSIM_DELIVERY_TILE] < 1e29f && mode_ev[BSIM_DELIVERY_TILE] > 0)
        out->cost_tile[1] = 1e3f * mode_best[BSIM_DELIVERY_TILE] / (float)mode_ev[BSIM_DELIVERY_TILE];
    return BSIM_OK;
}

int bsim_get_info(bsim_engine *eh, bsim_info *info)
{
    if (!eh || !info) return fail(BSIM_ERR_ARG, "invalid arguments");
    Engine &e = *H(eh);
    CK(cudaSetDevice(e.device));
    CK(cudaStreamSynchronize(e.stream));
    memset(info, 0, sizeof(*info));
    info->n_neurons = e.N;
    info->n_synapses = e.S;
    info->max_delay = e.D;
    info->n_instances = e.n_inst;
    info->n_classes = e.n_cls;
    info->n_pops = e.n_pops;
    unsigned long long ctr[2];
    CK(cudaMemcpy(ctr, e.a.step_ctr, sizeof(ctr), cudaMemcpyDeviceToHost));
    info->steps_done = (int64_t)ctr[0];
    info->events_total = ctr[1];
    info->device_bytes = e.device_bytes;
    info->grid_blocks = e.grid;
    info->block_threads = e.block;
    info->accumulate = e.opt.accumulate;
    info->delivery = e.opt.delivery;
    info->sm_count = e.sm_count;
    return BSIM_OK;
}

int bsim_get_qexp(bsim_engine *eh, int32_t *qexp)
{
    if (!eh || !qexp) return fail(BSIM_ERR_ARG, "invalid arguments");
    for (int i = 0; i < H(eh)->n_inst; i++) qexp[i] = H(eh)->qexp[i];
    return BSIM_OK;
}

int bsim_destroy(bsim_engine *eh)
{
    if (!eh) return BSIM_OK;
    free_engine(H(eh));
    return BSIM_OK;
}

const char *bsim_last_error(void) { return g_err.c_str(); }

}  // extern "C"
