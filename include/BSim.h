/*
 * BSim.h — the reference's user API for the single-GPU LIF_brian path, as a
 * header-only C++ front end over the bsim_b200 C ABI (bsim_b200.h).
 *
 * Programs written against the reference's include/BSim.h for this path —
 * Network, createPopulation<LIF_brian>, addNeuron, connect(weight, delay) and
 * SGSim(&net, dt).run(T) — compile against this header unchanged and run on
 * the B200 engine (link with -lbsim_b200). Names, argument meaning and output
 * files follow the reference:
 *   Network            src/net/Network.h:28-103, src/net/Network.cpp:118-150
 *   Population<T>      src/base/Population.h:15-203
 *   LIFENeuron         src/neuron/lif/LIFENeuron.h:9
 *   CompositeNeuron    src/base/CompositeNeuron.h:17-79 (LIF_brian, include/Neuron.h:31)
 *   SGSim              include/Simulator.h:21, src/sim/SingleGPUSimulator.cu:31-313
 *   FireInfo / logFireInfo  src/base/SimInfo.h:19-34, src/base/SimInfo.cpp:4-34
 *   getConstArray / getRandomArray  src/utils/utils.h:34-58
 *
 * Scope: LIF_brian (= IF_curr_exp) neurons and the Constant_spikes /
 * Poisson_spikes inputs with static delayed synapses on one GPU, fp32 (`real`
 * is float; building with USE_DOUBLE is an error). Other neuron types,
 * STSim/MGSim and the multi-GPU path are not provided.
 *
 * Differences from the reference, by design:
 *   - synapses whose delay rounds to 0 steps make run() fail with -4 (the
 *     reference CPU delivers them in the same cycle, its GPU build drops them);
 *   - run() returns the engine's status code instead of calling exit() on a
 *     CUDA error;
 *   - the single-synapse connect() returns NULL (no per-synapse object exists);
 *   - setting the environment variable BSIM_ACCUMULATE=ordered sums synaptic
 *     input in synapse creation order (bit-identical to the reference CPU
 *     simulator); the default exact int64 accumulation is order-independent;
 *   - BSIM_DELIVERY=tile (or pull) selects the delivery mode (same spikes);
 *   - Poisson_spikes draw from a generator seeded by BSIM_INPUT_SEED (default 1)
 *     instead of the clock, so runs are reproducible.
 */
#ifndef BSIM_B200_BSIM_H
#define BSIM_B200_BSIM_H

#ifdef USE_DOUBLE
#error "bsim_b200 implements the reference's float build; USE_DOUBLE is not supported"
#endif

#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>
#include <time.h>

#include <algorithm>
#include <map>
#include <string>
#include <vector>

#include "bsim_b200.h"

typedef float real;  // src/utils/constant.h:12-16 (float build)
typedef int ID;
const real ZERO = 1e-10;

enum Type { Constant = 0, Poisson = 1, Array, Decide, FFT, Mem, Max, LIFE, TJ, Static, TYPESIZE };
enum SpikeType { Excitatory = 0, Inhibitory = 1, SPIKETYPESIZE = 2 };

struct ArrayInfo {
    int size;
    void *data;
};
typedef std::map<std::string, ArrayInfo> FireInfo;

/* Writes <name>.<type>: one line of space-separated values (src/base/SimInfo.cpp:4-34). */
inline int logFireInfo(FireInfo log, std::string type, std::string name = "all")
{
    std::string filename = name.append(".").append(type);
    FILE *f = fopen(filename.c_str(), "w+");
    if (!f) {
        printf("ERROR: Open file %s failed\n", filename.c_str());
        return -1;
    }
    for (int j = 0; j < log[type].size; j++) {
        if (type == "Y") fprintf(f, "%f ", reinterpret_cast<real *>(log[type].data)[j]);
        else fprintf(f, "%d ", reinterpret_cast<int *>(log[type].data)[j]);
    }
    fprintf(f, "\n");
    fclose(f);
    return 0;
}

template <typename T>
T *getConstArray(T value, int size)
{
    T *res = new T[size];
    for (int i = 0; i < size; i++) res[i] = value;
    return res;
}

template <typename T>
T *getRandomArray(T range, int size)
{
    static bool seeded = false;
    if (!seeded) {
        srand((unsigned)time(NULL));
        seeded = true;
    }
    T *res = new T[size];
    for (int i = 0; i < size; i++) res[i] = static_cast<T>((double)rand() / RAND_MAX * (double)range);
    return res;
}

class SynapseBase;
class Network;

class NeuronBase {
public:
    NeuronBase() : _gid(-1) {}
    virtual ~NeuronBase() {}
    virtual Type getType() = 0;
    int getGlobalId() const { return _gid; }

protected:
    friend class Network;
    int _gid;  // position in the network (population order), set when the population joins
};

/* LIF neuron with exponential current synapses (src/neuron/lif/LIFENeuron.h:7-50).
 * Constructor arguments in the reference order, SI units. */
class LIFENeuron : public NeuronBase {
public:
    LIFENeuron(real v_init, real v_rest, real v_reset, real cm, real tau_m, real tau_refrac, real tau_syn_E,
               real tau_syn_I, real v_thresh, real i_offset)
    {
        real p[10] = {v_init, v_rest, v_reset, cm, tau_m, tau_refrac, tau_syn_E, tau_syn_I, v_thresh, i_offset};
        memcpy(_p, p, sizeof(_p));
    }
    virtual Type getType() { return LIFE; }
    const real *params() const { return _p; }
    const static Type type = LIFE;
    const static uint8_t kind = BSIM_NEURON_LIF;

private:
    real _p[10];
};

/* Spikes at a constant rate (src/neuron/constant/ConstantNeuron.h:15-50): fire_rate in
 * spikes per cycle, active from start_time until end_time (seconds). */
class ConstantNeuron : public NeuronBase {
public:
    ConstantNeuron(real fire_rate, real start_time = 0.0, real end_time = 1.0e9)
    {
        memset(_p, 0, sizeof(_p));
        _p[0] = fire_rate;
        _p[1] = start_time;
        _p[2] = end_time;
    }
    virtual Type getType() { return Constant; }
    void setRate(real rate) { _p[0] = rate; }
    void setStart(real time) { _p[1] = time; }
    void setEnd(real time) { _p[2] = time; }
    const real *params() const { return _p; }
    const static Type type = Constant;
    const static uint8_t kind = BSIM_NEURON_CONSTANT;

private:
    real _p[10];
};

/* Spikes with Poisson-distributed gaps (src/neuron/poisson/PoissonNeuron.h:18-58): rate is
 * the mean gap in cycles, refract the dead time after a spike (s), active for duration
 * seconds from start_time. Draws come from the engine's seeded generator
 * (BSIM_INPUT_SEED in the environment, default 1) instead of the system clock. */
class PoissonNeuron : public NeuronBase {
public:
    PoissonNeuron(real rate, real refract, real start_time = 0, real duration = 1000)
    {
        memset(_p, 0, sizeof(_p));
        _p[0] = rate;
        _p[1] = refract;
        _p[2] = start_time;
        _p[3] = duration;
    }
    virtual Type getType() { return Poisson; }
    const real *params() const { return _p; }
    const static Type type = Poisson;
    const static uint8_t kind = BSIM_NEURON_POISSON;

private:
    real _p[10];
};

class StaticSynapse {};  // synapse model tag: static weight + integer delay

/* A neuron model bundled with its synapse model; tau_syn_E / tau_syn_I pick the
 * decay applied to weights whose delay is not a multiple of dt
 * (src/base/CompositeNeuron.h:61-79). */
template <class Neuron, class Synapse>
class CompositeNeuron : public Neuron {
public:
    CompositeNeuron(const Neuron &templ, real tau_syn_E = 1e-3, real tau_syn_I = 1e-3)
        : Neuron(templ), _tau_syn_E(tau_syn_E), _tau_syn_I(tau_syn_I)
    {
    }
    real tauSynE() const { return _tau_syn_E; }
    real tauSynI() const { return _tau_syn_I; }

private:
    real _tau_syn_E, _tau_syn_I;
};

typedef CompositeNeuron<LIFENeuron, StaticSynapse> LIF_brian;
typedef CompositeNeuron<LIFENeuron, StaticSynapse> IF_curr_exp;
typedef CompositeNeuron<ConstantNeuron, StaticSynapse> Constant_spikes;  // include/Neuron.h:25
typedef CompositeNeuron<PoissonNeuron, StaticSynapse> Poisson_spikes;    // include/Neuron.h:26

class PopulationBase {
public:
    virtual ~PopulationBase() {}
    virtual int getNum() = 0;
    virtual NeuronBase *getNeuron(int idx) = 0;
    virtual Type getType() = 0;
    virtual const real *paramsOf(int idx) = 0;
    virtual uint8_t kindOf(int idx) = 0;
    virtual real tauOf(int idx, bool inhibitory) = 0;
};

template <class Neuron>
class Population : public PopulationBase {
public:
    Population(size_t N) : N(N) { neurons.reserve(N); }
    Population(size_t N, const Neuron &templ) : N(N), neurons(N, templ) {}
    int getNum() { return (int)N; }
    Type getType() { return Neuron::type; }
    NeuronBase *getNeuron(int idx) { return &neurons[idx]; }
    /* Appends a neuron with its own parameters (Population.h:158-168). */
    int addNeuron(Neuron templ)
    {
        neurons.push_back(templ);
        if (neurons.size() > N) {
            printf("Population overflow!!");
            N = neurons.size();
        }
        return (int)neurons.size() - 1;
    }
    const real *paramsOf(int idx) { return neurons[idx].params(); }
    uint8_t kindOf(int idx) { (void)idx; return Neuron::kind; }
    real tauOf(int idx, bool inh) { return inh ? neurons[idx].tauSynI() : neurons[idx].tauSynE(); }

private:
    size_t N;
    std::vector<Neuron> neurons;
};

class SynapseBase {};

/* The network under construction: populations plus a flat synapse list in
 * connect() order (no per-synapse objects). */
class Network {
public:
    Network() : maxDelaySteps(0), totalNeuronNum(0), totalSynapseNum(0), _maxDelay(0) {}
    ~Network()
    {
        for (PopulationBase *p : pPopulations) delete p;
    }

    template <class Neuron>
    Population<Neuron> *createPopulation(int id, int num, Neuron templ, bool empty = false)
    {
        (void)id;
        return createPopulation(num, templ, empty);
    }

    template <class Neuron>
    Population<Neuron> *createPopulation(int num, Neuron templ, bool empty = false)
    {
        Population<Neuron> *p = empty ? new Population<Neuron>(num) : new Population<Neuron>(num, templ);
        pPopulations.push_back(p);
        return p;
    }

    /* All-to-all with one weight and delay (Network.h:146-174). */
    template <class N1, class N2>
    int connect(Population<N1> *pSrc, Population<N2> *pDst, real weight, real delay, SpikeType type)
    {
        int count = 0;
        for (int i = 0; i < pSrc->getNum(); i++)
            for (int j = 0; j < pDst->getNum(); j++, count++)
                connect(pSrc->getNeuron(i), pDst->getNeuron(j), weight, delay, type, 0.0, false);
        return count;
    }

    /* All-to-all with per-pair arrays, source-major (Network.h:176-209); type may be NULL. */
    template <class N1, class N2>
    int connect(Population<N1> *pSrc, Population<N2> *pDst, real *weight, real *delay, SpikeType *type, int size)
    {
        const int ns = pSrc->getNum(), nd = pDst->getNum();
        if (size != ns * nd) {
            fprintf(stderr, "connect: size %d != %d x %d\n", size, ns, nd);
            abort();
        }
        for (int i = 0; i < size; i++)
            connect(pSrc->getNeuron(i / nd), pDst->getNeuron(i % nd), weight[i], delay[i],
                    type ? type[i] : Excitatory, 0.0, false);
        return size;
    }

    template <class N1, class N2>
    int connectOne2One(Population<N1> *pSrc, Population<N2> *pDst, real *weight, real *delay, SpikeType *type,
                       int size)
    {
        for (int i = 0; i < size; i++)
            connect(pSrc->getNeuron(i), pDst->getNeuron(i), weight[i], delay[i], type ? type[i] : Excitatory,
                    0.0, false);
        return size;
    }

    /* One synapse (Network.cpp:118-150). tau != 0 overrides the target's tau_syn. */
    SynapseBase *connect(NeuronBase *pSrc, NeuronBase *pDst, real weight, real delay, SpikeType type = Excitatory,
                         real tau = 0, bool store = true)
    {
        (void)store;
        _src.push_back(pSrc);
        _dst.push_back(pDst);
        _w.push_back(weight);
        _d.push_back(delay);
        _type.push_back((uint8_t)type);
        _tau.push_back(tau);
        if (delay > _maxDelay) _maxDelay = delay;
        totalSynapseNum++;
        return NULL;
    }

    /* By (population index, neuron index); the spike type follows the weight's sign (Network.cpp:236-284). */
    int connect(int popSrc, int nSrc, int popDst, int nDst, real weight, real delay, real tau = 0)
    {
        if (popSrc >= (int)pPopulations.size() || popDst >= (int)pPopulations.size()) return -1;
        connect(pPopulations[popSrc]->getNeuron(nSrc), pPopulations[popDst]->getNeuron(nDst), weight, delay,
                weight < 0.0 ? Inhibitory : Excitatory, tau, false);
        return 0;
    }

    /* Flattens the network for the engine: per-neuron parameters in population
     * order and synapses in connect() order with StaticSynapse::reset applied
     * (src/synapse/static/StaticSynapse.cpp:43-54). Returns 0 or a BSIM_ERR_* code. */
    int flatten(real dt, std::vector<float> &params, std::vector<int32_t> &pop, std::vector<int32_t> &src,
                std::vector<int32_t> &dst, std::vector<float> &weight, std::vector<int32_t> &delay_steps,
                std::vector<uint8_t> *kind = NULL)
    {
        std::map<NeuronBase *, std::pair<int, int>> where;  // neuron -> (population, index)
        int g = 0;
        params.clear();
        pop.clear();
        if (kind) kind->clear();
        for (size_t p = 0; p < pPopulations.size(); p++) {
            PopulationBase *pp = pPopulations[p];
            for (int i = 0; i < pp->getNum(); i++, g++) {
                NeuronBase *nb = pp->getNeuron(i);
                nb->_gid = g;
                where[nb] = std::make_pair((int)p, i);
                const real *q = pp->paramsOf(i);
                params.insert(params.end(), q, q + 10);
                pop.push_back((int32_t)p);
                if (kind) kind->push_back(pp->kindOf(i));
            }
        }
        totalNeuronNum = g;
        const size_t s = _src.size();
        src.resize(s);
        dst.resize(s);
        std::vector<float> tau(s), d(s);
        for (size_t k = 0; k < s; k++) {
            if (_src[k]->_gid < 0 || _dst[k]->_gid < 0) return BSIM_ERR_ARG;
            src[k] = _src[k]->_gid;
            dst[k] = _dst[k]->_gid;
            if (fabsf(_tau[k]) > ZERO) {
                tau[k] = _tau[k];
            } else {
                std::pair<int, int> w = where[_dst[k]];
                tau[k] = pPopulations[w.first]->tauOf(w.second, _type[k] == Inhibitory);
            }
            d[k] = _d[k];
        }
        weight.resize(s);
        delay_steps.resize(s);
        int rc = bsim_synapse_reset(d.data(), _w.data(), tau.data(), (int64_t)s, dt, delay_steps.data(),
                                    weight.data());
        maxDelaySteps = (int)roundf(_maxDelay / dt);
        return rc;
    }

    std::vector<PopulationBase *> pPopulations;
    int maxDelaySteps;
    int totalNeuronNum;
    int totalSynapseNum;

private:
    std::vector<NeuronBase *> _src, _dst;
    std::vector<real> _w, _d, _tau;
    std::vector<uint8_t> _type;
    real _maxDelay;
};

class SimulatorBase {
public:
    SimulatorBase(Network *network, real dt) : network(network), dt(dt) {}
    virtual ~SimulatorBase() {}
    virtual int run(real time, FireInfo &log) = 0;
    virtual int reset() { return 0; }

    /* Runs and writes GFire.count (src/base/SimulatorBase.cpp:29-37). */
    int run(real time)
    {
        FireInfo fire_info;
        ArrayInfo zero = {0, NULL};
        fire_info["count"] = zero;
        int ret = run(time, fire_info);
        logFireInfo(fire_info, "count", "GFire");
        free(fire_info["count"].data);
        return ret;
    }

protected:
    Network *network;
    real dt;
};

/* SingleGPUSimulator (SGSim) on the B200 engine. run(time, log) builds the
 * engine, runs round(time/dt) cycles, writes GSim.info and fills log["count"]
 * (spikes per neuron). Compiled with -DLOG_DATA it also writes GSim.log (fired
 * ids per cycle, ascending) and g_v.data / g_ie.data / g_ii.data ("%.10lf \t"
 * per neuron per cycle), the reference's LOG_DATA files (SingleGPUSimulator.cu:150-242). */
class SingleGPUSimulator : public SimulatorBase {
public:
    SingleGPUSimulator(Network *network, real dt) : SimulatorBase(network, dt) {}
    using SimulatorBase::run;

    virtual int run(real time, FireInfo &log)
    {
        const int sim_cycle = (int)round(time / dt);
        std::vector<float> params, weight;
        std::vector<int32_t> pop, src, dst, delay;
        std::vector<uint8_t> kind;
        int rc = network->flatten(dt, params, pop, src, dst, weight, delay, &kind);
        if (rc != BSIM_OK) return rc;
        FILE *info_file = fopen("GSim.info", "w+");
        if (!info_file) {
            printf("ERROR: Open file GSim.info failed\n");
            return -1;
        }
        bsim_options opt;
        bsim_options_default(&opt);
        const char *acc = getenv("BSIM_ACCUMULATE");
        if (acc && strcmp(acc, "ordered") == 0) opt.accumulate = BSIM_ACC_ORDERED;
        const char *del = getenv("BSIM_DELIVERY");  // push (default), tile or pull
        if (del && strcmp(del, "tile") == 0) opt.delivery = BSIM_DELIVERY_TILE;
        if (del && strcmp(del, "pull") == 0) opt.delivery = BSIM_DELIVERY_PULL;
        const int64_t n = (int64_t)pop.size();
        const char *seed_env = getenv("BSIM_INPUT_SEED");
        const uint64_t seed = seed_env ? strtoull(seed_env, NULL, 10) : 1;
        int n_types = 0;
        for (int k = 0; k < 3; k++) n_types += std::find(kind.begin(), kind.end(), (uint8_t)k) != kind.end();
        bsim_engine *e = NULL;
        rc = bsim_create_mixed(params.data(), kind.data(), n, pop.data(), NULL, src.data(), dst.data(),
                               weight.data(), delay.data(), (int64_t)src.size(), dt, seed, &opt, &e);
        if (rc != BSIM_OK) {
            fprintf(stderr, "bsim_create_mixed: %s\n", bsim_last_error());
            fclose(info_file);
            return rc;
        }
        bsim_info inf;
        bsim_get_info(e, &inf);
        fprintf(info_file, "NeuronTypeNum: %d, SynapseTypeNum: %d\n", n_types, 1);
        fprintf(info_file, "NeuronNum: %lld, SynapseNum: %lld\n", (long long)n, (long long)src.size());
        fprintf(info_file, "MAX_DELAY: %d\n", inf.max_delay);
        fprintf(info_file, "Start runing for %d cycles\n", sim_cycle);
        struct timeval ts, te;
        gettimeofday(&ts, NULL);
#ifdef LOG_DATA
        rc = run_logged(e, sim_cycle, n);
#else
        rc = bsim_run(e, sim_cycle);
#endif
        gettimeofday(&te, NULL);
        if (rc != BSIM_OK) fprintf(stderr, "bsim_run: %s\n", bsim_last_error());
        long us = (te.tv_sec - ts.tv_sec) * 1000000L + (te.tv_usec - ts.tv_usec);
        fprintf(info_file, "Simulation finesed in %ld:%ld:%ld.%06lds\n", us / 3600000000L, (us / 60000000L) % 60,
                (us / 1000000L) % 60, us % 1000000L);
        fclose(info_file);
        if (rc == BSIM_OK && log.find("count") != log.end()) {
            int *rate = (int *)malloc(sizeof(int) * n);
            rc = bsim_read_fire_count(e, rate);
            log["count"].size = (int)n;
            log["count"].data = rate;
        }
        bsim_destroy(e);
        return rc;
    }

private:
#ifdef LOG_DATA
    // The reference's LOG_DATA files (SingleGPUSimulator.cu:150-242): per cycle one line
    // of fired ids (GSim.log; ascending here, in atomic order there) and one line of
    // "%.10lf \t" values per neuron for v, i_E, i_I and the synaptic input the cycle
    // consumed. The engine records spikes and the state trace on the device inside the
    // step; the host reads them back once per chunk of cycles (sized to ~256 MB of
    // buffers), not once per cycle.
    int run_logged(bsim_engine *e, int cycles, int64_t n)
    {
        const char *names[6] = {"GSim.log", "g_v.data", "g_ie.data", "g_ii.data", "g_input_e.data",
                                "g_input_i.data"};
        FILE *f[6];
        for (int k = 0; k < 6; k++) f[k] = fopen(names[k], "w+");
        int rc = BSIM_OK;
        for (int k = 0; k < 6; k++)
            if (!f[k]) rc = -1;
        const int64_t per_cycle = 4 * (6 * n + 2);
        const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(cycles, (256LL << 20) / per_cycle));
        std::vector<float> tr(5 * chunk * n);
        std::vector<int64_t> off(chunk + 1);
        std::vector<int32_t> ids(chunk * n);
        for (int t0 = 0; t0 < cycles && rc == BSIM_OK; t0 += (int)chunk) {
            const int64_t k = std::min<int64_t>(chunk, cycles - t0);
            rc = bsim_record(e, k, k * n);
            if (rc == BSIM_OK) rc = bsim_trace(e, k, 0, n);
            if (rc == BSIM_OK) rc = bsim_run(e, k);
            int64_t ns = 0, nt = 0;
            if (rc == BSIM_OK) rc = bsim_read_raster(e, off.data(), ids.data(), k * n, &ns);
            if (rc == BSIM_OK)
                rc = bsim_read_trace(e, tr.data(), tr.data() + k * n, tr.data() + 2 * k * n, tr.data() + 3 * k * n,
                                     tr.data() + 4 * k * n, &nt);
            if (rc != BSIM_OK) break;
            for (int64_t c = 0; c < k; c++) {
                for (int64_t i = (c < ns ? off[c] : 0); i < (c < ns ? off[c + 1] : 0); i++) fprintf(f[0], "%d ", ids[i]);
                fprintf(f[0], "\n");
                for (int q = 0; q < 5; q++) {
                    const float *row = tr.data() + (int64_t)q * k * n + c * n;
                    if (c < nt)
                        for (int64_t i = 0; i < n; i++) fprintf(f[1 + q], "%.10lf \t", (double)row[i]);
                    fprintf(f[1 + q], "\n");
                }
            }
        }
        for (int k = 0; k < 6; k++)
            if (f[k]) fclose(f[k]);
        return rc;
    }
#endif
};

typedef SingleGPUSimulator SGSim;

#endif /* BSIM_B200_BSIM_H */
