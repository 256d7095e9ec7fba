/*
 * TEST INFRASTRUCTURE ONLY. Body of the oracle, included twice by lif_oracle.c:
 * once with REAL=float (suffix _f32) and once with REAL=double (suffix _f64),
 * mirroring the reference's `real` typedef (src/utils/constant.h:12-16).
 *
 * Required macros: REAL, SFX(name), R_EXP (exp for REAL), R_FABS, R_ROUND.
 * Built with -ffp-contract=off so that every product and sum is rounded to
 * REAL on its own, as in the reference's x86-64 build (SSE, no FMA).
 */

/* LIFENeuron::reset (src/neuron/lif/LIFENeuron.cpp:68-112), one neuron at a time.
 * ZERO = 1e-10 is the reference constant of src/utils/constant.h:20. */
int SFX(oracle_lif_reset)(const REAL *params, int64_t n, REAL dt, REAL *fold, int32_t *refrac_time)
{
    const REAL ZERO_ = (REAL)1e-10;
    if (n < 0 || (n > 0 && (!params || !fold || !refrac_time))) return -1;
    for (int64_t i = 0; i < n; i++) {
        const REAL *p = params + i * ORACLE_NPARAM;
        REAL v_init = p[0], v_rest = p[1], v_reset = p[2], cm = p[3], tau_m = p[4];
        REAL tau_refrac = p[5], tau_syn_E = p[6], tau_syn_I = p[7], v_thresh = p[8], i_offset = p[9];
        REAL rm = (REAL)1.0;
        if (R_FABS(cm) > ZERO_) rm = tau_m / cm;
        REAL Cm = tau_m > 0 ? (REAL)R_EXP(-dt / tau_m) : (REAL)0.0;
        REAL CE = tau_syn_E > 0 ? (REAL)R_EXP(-dt / tau_syn_E) : (REAL)0.0;
        REAL CI = tau_syn_I > 0 ? (REAL)R_EXP(-dt / tau_syn_I) : (REAL)0.0;
        REAL v_tmp = i_offset * rm + v_rest;
        v_tmp = v_tmp * ((REAL)1 - Cm);
        REAL C_E = rm * tau_syn_E / (tau_syn_E - tau_m);
        REAL C_I = rm * tau_syn_I / (tau_syn_I - tau_m);
        C_E = C_E * (CE - Cm);
        C_I = C_I * (CI - Cm);
        REAL *f = fold + i * ORACLE_NFOLD;
        f[0] = v_init; f[1] = CI; f[2] = CE; f[3] = C_I; f[4] = C_E; f[5] = v_tmp;
        f[6] = 0; f[7] = 0; f[8] = v_thresh; f[9] = v_reset; f[10] = Cm;
        refrac_time[i] = (int32_t)(tau_refrac / dt);
    }
    return 0;
}

/* StaticSynapse::reset (src/synapse/static/StaticSynapse.cpp:43-54): delay in
 * seconds -> whole steps (round), and the weight decay applied when the delay
 * is not a multiple of dt. The reference calls expf() here in both builds. */
int SFX(oracle_syn_reset)(const REAL *delay_s, const REAL *weight, const REAL *tau_syn,
                          int64_t s, REAL dt, int32_t *delay_steps, REAL *weight_out)
{
    const REAL ZERO_ = (REAL)1e-10;
    if (s < 0 || (s > 0 && (!delay_s || !weight || !tau_syn || !delay_steps || !weight_out))) return -1;
    for (int64_t i = 0; i < s; i++) {
        int32_t st = (int32_t)R_ROUND(delay_s[i] / dt);
        REAL rem = delay_s[i] - dt * (REAL)st;
        REAL w = weight[i];
        if (R_FABS(tau_syn[i]) > ZERO_ && R_FABS(rem) > ZERO_) {
            REAL c1 = (REAL)expf((float)(-rem / tau_syn[i]));
            w = w * c1;
        }
        delay_steps[i] = st;
        weight_out[i] = w;
    }
    return 0;
}

static int SFX(cmp_i64)(const void *a, const void *b)
{
    int64_t x = *(const int64_t *)a, y = *(const int64_t *)b;
    return (x > y) - (x < y);
}

/* SingleThreadSimulator::run (src/sim/SingleThreadSimulator.cpp:21-183).
 *
 * Each cycle runs Network::update (src/net/Network.cpp:308-330): every neuron in
 * population order (LIFENeuron::update), then every synapse in creation order
 * (StaticSynapse::update). A spike of neuron s at cycle t pushes `delay_steps`
 * onto each out-synapse's queue (NeuronBase::fire -> StaticSynapse::recv); the
 * queue front is delivered when it reaches 0, i.e. in the synapse phase of cycle
 * t + delay, and is consumed by the target's update at cycle t + delay + 1.
 *
 * Restated without per-synapse queues: in the synapse phase of cycle t, synapse
 * k delivers iff its source fired at cycle t - delay(k). The delivering synapse
 * ids are sorted, so the per-target sums are formed in creation order exactly as
 * the reference's loop over pSynapses forms them (each synapse delivers at most
 * once per cycle because a neuron fires at most once per cycle).
 *
 * Delays of 0 steps are rejected (-2): the reference CPU delivers them in the
 * same cycle while the reference GPU build drops them (BuildNetwork.cpp:108-110).
 */
int SFX(oracle_run)(const REAL *params, int64_t n,
                    const int32_t *src, const int32_t *dst, const REAL *weight,
                    const int32_t *delay_steps, int64_t s, REAL dt, int64_t steps,
                    int acc_mode, const int32_t *qexp_per_neuron, oracle_out *out)
{
    if (n <= 0 || s < 0 || steps < 0 || !params || !out) return -1;
    if (acc_mode != ORACLE_ACC_SEQUENTIAL && acc_mode != ORACLE_ACC_FIXED) return -1;
    if (acc_mode == ORACLE_ACC_FIXED && !qexp_per_neuron) return -1;
    int32_t D = 1;
    for (int64_t k = 0; k < s; k++) {
        if (src[k] < 0 || src[k] >= n || dst[k] < 0 || dst[k] >= n) return -3;
        if (delay_steps[k] < 1) return -2;
        if (delay_steps[k] > D) D = delay_steps[k];
    }
    const int32_t R = D + 1; /* ring of fired lists, one per cycle in the delay window */

    REAL *fold = (REAL *)malloc(sizeof(REAL) * ORACLE_NFOLD * (size_t)n);
    int32_t *rtime = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
    int32_t *rstep = (int32_t *)calloc((size_t)n, sizeof(int32_t));
    REAL *synE = (REAL *)calloc((size_t)n, sizeof(REAL));
    REAL *synI = (REAL *)calloc((size_t)n, sizeof(REAL));
    int64_t *accE = (int64_t *)calloc((size_t)n, sizeof(int64_t));
    int64_t *accI = (int64_t *)calloc((size_t)n, sizeof(int64_t));
    int64_t *off = (int64_t *)calloc((size_t)n * D + 1, sizeof(int64_t));
    int64_t *ids = (int64_t *)malloc(sizeof(int64_t) * (size_t)(s > 0 ? s : 1));
    int32_t *ring = (int32_t *)malloc(sizeof(int32_t) * (size_t)n * R);
    int64_t *ring_n = (int64_t *)calloc((size_t)R, sizeof(int64_t));
    int64_t ev_cap = 1024;
    int64_t *ev = (int64_t *)malloc(sizeof(int64_t) * (size_t)ev_cap);
    REAL *vtmp_base = NULL, *vtmp_alt = NULL; /* square-wave drive: v_tmp of each phase */
    /* input-drive neurons: Constant {start_cycle, end_cycle, fire_count},
     * Poisson {fire_cycle, end_cycle, refrac_step}, and each neuron's draw id */
    int32_t *dslot = NULL;
    int64_t *draw_id = NULL;
    const uint8_t *kind = out->kind;
    int rc = 0;
    if (!fold || !rtime || !rstep || !synE || !synI || !accE || !accI || !off || !ids || !ring || !ring_n || !ev) {
        rc = -4;
        goto done;
    }
    SFX(oracle_lif_reset)(params, n, dt, fold, rtime);
    if (kind) {
        dslot = (int32_t *)calloc((size_t)n * 3, sizeof(int32_t));
        draw_id = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
        if (!dslot || !draw_id || o_tables()) { rc = -4; goto done; }
        /* Poisson draws are keyed by (seed, id - first id of the neuron's network, cycle) */
        if (out->instance) {
            int32_t ninst = 1;
            for (int64_t j = 0; j < n; j++) {
                if (out->instance[j] < 0) { rc = -1; goto done; }
                if (out->instance[j] >= ninst) ninst = out->instance[j] + 1;
            }
            int64_t *first = (int64_t *)malloc(sizeof(int64_t) * (size_t)ninst);
            if (!first) { rc = -4; goto done; }
            for (int32_t g = 0; g < ninst; g++) first[g] = -1;
            for (int64_t j = 0; j < n; j++) {
                if (first[out->instance[j]] < 0) first[out->instance[j]] = j;
                draw_id[j] = j - first[out->instance[j]];
            }
            free(first);
        } else {
            for (int64_t j = 0; j < n; j++) draw_id[j] = j;
        }
        for (int64_t j = 0; j < n; j++) {
            const REAL *p = params + j * ORACLE_NPARAM;
            int32_t *ds = dslot + 3 * j;
            if (kind[j] == 1) {
                /* ConstantNeuron::reset (src/neuron/constant/ConstantNeuron.cpp:55-62) */
                ds[0] = R_CYCLE(p[1] / dt);
                ds[1] = R_CYCLE(p[2] / dt);
                ds[2] = 0;
            } else if (kind[j] == 2) {
                /* PoissonNeuron::reset (src/neuron/poisson/PoissonNeuron.cpp:35-44) */
                float rate = (float)p[0];
                if (!(rate >= 0.0f && rate < 16777216.0f)) { rc = -1; goto done; }
                int64_t fc = (int64_t)R_CYCLE(p[2] / dt) +
                             o_poisson_draw(o_poisson_key(out->input_seed, draw_id[j], -1), rate);
                ds[0] = fc > INT32_MAX ? INT32_MAX : (int32_t)fc;
                ds[1] = R_CYCLE((p[2] + p[3]) / dt);
                ds[2] = R_CYCLE(p[1] / dt);
            } else if (kind[j] != 0) {
                rc = -1;
                goto done;
            }
        }
    }
    if (out->params_alt && out->half_period > 0) {
        REAL *fa = (REAL *)malloc(sizeof(REAL) * ORACLE_NFOLD * (size_t)n);
        int32_t *ra = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
        vtmp_base = (REAL *)malloc(sizeof(REAL) * (size_t)n);
        vtmp_alt = (REAL *)malloc(sizeof(REAL) * (size_t)n);
        if (!fa || !ra || !vtmp_base || !vtmp_alt) {
            free(fa); free(ra); free(vtmp_base); free(vtmp_alt);
            rc = -4;
            goto done;
        }
        SFX(oracle_lif_reset)((const REAL *)out->params_alt, n, dt, fa, ra);
        for (int64_t j = 0; j < n; j++) {
            vtmp_base[j] = fold[j * ORACLE_NFOLD + 5];
            vtmp_alt[j] = fa[j * ORACLE_NFOLD + 5];
        }
        free(fa);
        free(ra);
    }

    /* Synapse ids grouped by (source, delay), creation order inside a group. */
    for (int64_t k = 0; k < s; k++) off[(int64_t)src[k] * D + (delay_steps[k] - 1) + 1]++;
    for (int64_t i = 0; i < (int64_t)n * D; i++) off[i + 1] += off[i];
    {
        int64_t *cur = (int64_t *)malloc(sizeof(int64_t) * (size_t)n * D);
        if (!cur) { rc = -4; goto done; }
        memcpy(cur, off, sizeof(int64_t) * (size_t)n * D);
        for (int64_t k = 0; k < s; k++) ids[cur[(int64_t)src[k] * D + delay_steps[k] - 1]++] = k;
        free(cur);
    }
    if (out->fire_count) memset(out->fire_count, 0, sizeof(int32_t) * (size_t)n);
    if (out->raster_off && out->record_steps > 0) out->raster_off[0] = 0;
    int64_t raster_pos = 0;

    for (int64_t t = 0; t < steps; t++) {
        /* ---- neuron phase: LIFENeuron::update (LIFENeuron.cpp:114-160) ---- */
        const int32_t slot = (int32_t)(t % R);
        int32_t *fired_list = ring + (int64_t)slot * n;
        int64_t nf = 0;
        if (vtmp_alt && (t % out->half_period) == 0) {
            const REAL *src_vt = ((t / out->half_period) & 1) ? vtmp_alt : vtmp_base;
            for (int64_t j = 0; j < n; j++) fold[j * ORACLE_NFOLD + 5] = src_vt[j];
        }
        for (int64_t j = 0; j < n; j++) {
            REAL *f = fold + j * ORACLE_NFOLD;
            REAL in_E, in_I;
            if (acc_mode == ORACLE_ACC_FIXED) {
                REAL sc = (REAL)ldexp(1.0, -qexp_per_neuron[j]);
                in_E = (REAL)accE[j] * sc;
                in_I = (REAL)accI[j] * sc;
                accE[j] = 0;
                accI[j] = 0;
            } else {
                in_E = synE[j];
                in_I = synI[j];
            }
            int fired = 0;
            if (kind && kind[j] == 1) {
                /* update_constant_neuron (src/neuron/constant/constant.cu:18-22) */
                int32_t *ds = dslot + 3 * j;
                REAL rate = params[j * ORACLE_NPARAM];
                if ((int32_t)t < ds[1] && (REAL)((int32_t)t - ds[0]) * rate > (REAL)ds[2]) {
                    fired = 1;
                    ds[2]++;
                }
            } else if (kind && kind[j] == 2) {
                /* update_poisson_neuron + reset_poisson_neuron (src/neuron/poisson/poisson.cu:29-31, 9-15) */
                int32_t *ds = dslot + 3 * j;
                if ((int32_t)t == ds[0] && (int32_t)t <= ds[1]) {
                    fired = 1;
                    float rate = (float)params[j * ORACLE_NPARAM];
                    int64_t nxt = (int64_t)ds[0] + 1 +
                                  o_poisson_draw(o_poisson_key(out->input_seed, draw_id[j], ds[0]), rate) + ds[2];
                    ds[0] = nxt > INT32_MAX ? INT32_MAX : (int32_t)nxt;
                }
            } else if (rstep[j] > 0) {
                --rstep[j];
            } else {
                REAL vm = f[10] * f[0] + f[5] + f[7] * f[4] + f[6] * f[3];
                f[7] = f[2] * f[7];
                f[6] = f[1] * f[6];
                if (vm >= f[8]) {
                    fired = 1;
                    rstep[j] = rtime[j] - 1;
                    vm = f[9];
                } else {
                    f[7] += in_E;
                    f[6] += in_I;
                }
                f[0] = vm;
            }
            synE[j] = 0;
            synI[j] = 0;
            if (fired) {
                fired_list[nf++] = (int32_t)j;
                if (out->fire_count) out->fire_count[j]++;
            }
        }
        ring_n[slot] = nf;
        if (out->spikes_per_step) out->spikes_per_step[t] = nf;
        if (t < out->record_steps) {
            if (out->raster_ids && out->raster_off) {
                if (raster_pos + nf > out->raster_cap) { rc = -5; goto done; }
                memcpy(out->raster_ids + raster_pos, fired_list, sizeof(int32_t) * (size_t)nf);
                raster_pos += nf;
                out->raster_off[t + 1] = raster_pos;
            }
            if (out->v_trace && out->rec_ids) {
                REAL *vt = (REAL *)out->v_trace + t * out->n_rec;
                for (int64_t r = 0; r < out->n_rec; r++) vt[r] = fold[(int64_t)out->rec_ids[r] * ORACLE_NFOLD];
            }
        }

        /* ---- synapse phase: StaticSynapse::update over pSynapses ---- */
        int64_t ne = 0;
        for (int32_t d = 1; d <= D && d <= t; d++) {
            const int32_t sl = (int32_t)((t - d) % R);
            const int32_t *fl = ring + (int64_t)sl * n;
            for (int64_t q = 0; q < ring_n[sl]; q++) {
                int64_t g = (int64_t)fl[q] * D + (d - 1);
                int64_t a = off[g], b = off[g + 1];
                if (ne + (b - a) > ev_cap) {
                    while (ne + (b - a) > ev_cap) ev_cap *= 2;
                    int64_t *nev = (int64_t *)realloc(ev, sizeof(int64_t) * (size_t)ev_cap);
                    if (!nev) { rc = -4; goto done; }
                    ev = nev;
                }
                for (int64_t e = a; e < b; e++) ev[ne++] = ids[e];
            }
        }
        if (out->events_per_step) out->events_per_step[t] = ne;
        if (acc_mode == ORACLE_ACC_SEQUENTIAL) {
            qsort(ev, (size_t)ne, sizeof(int64_t), SFX(cmp_i64));
            for (int64_t e = 0; e < ne; e++) {
                int64_t k = ev[e];
                REAL w = weight[k];
                /* LIFENeuron::recv: sign routes to the E or I accumulator */
                if (w >= 0) synE[dst[k]] += w;
                else synI[dst[k]] += w;
            }
        } else {
            for (int64_t e = 0; e < ne; e++) {
                int64_t k = ev[e];
                int32_t j = dst[k];
                REAL w = weight[k];
                REAL sc = (REAL)ldexp(1.0, qexp_per_neuron[j]);
                int64_t c = (int64_t)llrint((double)(w * sc));
                if (w >= 0) accE[j] = (int64_t)((uint64_t)accE[j] + (uint64_t)c);
                else accI[j] = (int64_t)((uint64_t)accI[j] + (uint64_t)c);
            }
        }
    }
    if (out->final_state) {
        REAL *fs = (REAL *)out->final_state;
        for (int64_t j = 0; j < n; j++) {
            if (kind && kind[j] != 0) {
                /* drive neurons: rate, then their three counters */
                fs[j * 4 + 0] = params[j * ORACLE_NPARAM];
                fs[j * 4 + 1] = (REAL)dslot[3 * j];
                fs[j * 4 + 2] = (REAL)dslot[3 * j + 1];
                fs[j * 4 + 3] = (REAL)dslot[3 * j + 2];
                continue;
            }
            fs[j * 4 + 0] = fold[j * ORACLE_NFOLD + 0];
            fs[j * 4 + 1] = fold[j * ORACLE_NFOLD + 7];
            fs[j * 4 + 2] = fold[j * ORACLE_NFOLD + 6];
            fs[j * 4 + 3] = (REAL)rstep[j];
        }
    }
done:
    free(dslot); free(draw_id);
    free(vtmp_base); free(vtmp_alt);
    free(fold); free(rtime); free(rstep); free(synE); free(synI); free(accE); free(accI);
    free(off); free(ids); free(ring); free(ring_n); free(ev);
    return rc;
}
