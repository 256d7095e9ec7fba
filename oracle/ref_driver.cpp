/*
 * TEST INFRASTRUCTURE ONLY. Driver that runs the REFERENCE's own CPU simulator
 * path, compiled from the reference sources by oracle/Makefile into oracle/_ref/.
 *
 * It builds a network through the reference's public API — createPopulation
 * with empty=true + Population::addNeuron for per-neuron parameters
 * (src/net/Network.h:120-144, src/base/Population.h:158-168) and the
 * single-synapse Network::connect (src/net/Network.cpp:118-150) in the file's
 * synapse creation order — then runs the loop of SingleThreadSimulator::run
 * (src/sim/SingleThreadSimulator.cpp:84-100): SimulatorBase::reset() once, then
 * Network::update + Network::monitor per cycle, recording SimInfo::fired and
 * SimInfo::input exactly as the reference's LOG_DATA build writes them.
 *
 * Usage: ref_driver <net.bin> <out.bin> [--no-record]
 * File formats are documented in tests/netio.py.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <vector>

#include "include/Neuron.h"
#include "src/net/Network.h"
#include "src/sim/SingleThreadSimulator.h"

typedef CompositeNeuron<LIFENeuron, StaticSynapse> LIFBrianRef; /* include/Neuron.h:31 */

template <typename T>
static bool rd(FILE *f, T *p, size_t n)
{
    return fread(p, sizeof(T), n, f) == n;
}

int main(int argc, char **argv)
{
    if (argc < 3) {
        fprintf(stderr, "usage: %s net.bin out.bin [--no-record]\n", argv[0]);
        return 2;
    }
    bool record = !(argc > 3 && strcmp(argv[3], "--no-record") == 0);
    FILE *f = fopen(argv[1], "rb");
    if (!f) return 3;
    char magic[4];
    int64_t hdr[6];
    double dt;
    if (!rd(f, magic, 4) || memcmp(magic, "BSNT", 4) != 0) return 4;
    if (!rd(f, hdr, 6) || !rd(f, &dt, 1)) return 4;
    int64_t n = hdr[0], s = hdr[1], steps = hdr[2], rec_steps = hdr[3], n_pop = hdr[4], n_rec = hdr[5];
    std::vector<int64_t> pop_size(n_pop);
    std::vector<double> pop_tau(2 * n_pop), params(10 * n), w(s), d(s);
    std::vector<int32_t> src(s), dst(s), rec(n_rec);
    std::vector<uint8_t> type(s);
    if (!rd(f, pop_size.data(), n_pop) || !rd(f, pop_tau.data(), 2 * n_pop) || !rd(f, params.data(), 10 * n) ||
        !rd(f, src.data(), s) || !rd(f, dst.data(), s) || !rd(f, w.data(), s) || !rd(f, d.data(), s) ||
        !rd(f, type.data(), s) || !rd(f, rec.data(), n_rec))
        return 5;
    fclose(f);

    Network net;
    std::vector<NeuronBase *> neuron(n);
    int64_t g = 0;
    for (int64_t p = 0; p < n_pop; p++) {
        const double *q = &params[10 * g];
        LIFBrianRef templ(LIFENeuron(q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7], q[8], q[9]),
                          (real)pop_tau[2 * p], (real)pop_tau[2 * p + 1]);
        Population<LIFBrianRef> *pop = net.createPopulation((int)pop_size[p], templ, true);
        for (int64_t i = 0; i < pop_size[p]; i++, g++) {
            const double *r = &params[10 * g];
            pop->addNeuron(LIFBrianRef(LIFENeuron(r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7], r[8], r[9]),
                                       (real)pop_tau[2 * p], (real)pop_tau[2 * p + 1]));
        }
        for (int64_t i = 0; i < pop_size[p]; i++) neuron[g - pop_size[p] + i] = pop->getNeuron((int)i);
    }
    if (g != n) return 6;
    for (int64_t k = 0; k < s; k++)
        net.connect(neuron[src[k]], neuron[dst[k]], (real)w[k], (real)d[k],
                    type[k] ? Inhibitory : Excitatory, 0.0, false);

    SingleThreadSimulator sim(&net, (real)dt); /* STSim, include/Simulator.h:19 */
    sim.reset();

    std::vector<int64_t> raster_n;
    std::vector<int32_t> raster;
    std::vector<double> vtrace;
    std::vector<double> last(5 * n, 0.0);
    SimInfo info;
    info.currCycle = 0;
    info.dt = (real)dt;
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    for (int64_t c = 0; c < steps; c++) {
        info.currCycle = (int)c;
        info.fired.clear();
        info.input.clear();
        net.update(info);
        net.monitor(info);
        if (record && c < rec_steps) {
            int64_t cnt = 0;
            for (int64_t i = 0; i < (int64_t)info.fired.size(); i++)
                if (info.fired[i]) { raster.push_back((int32_t)i); cnt++; }
            raster_n.push_back(cnt);
            for (int64_t r = 0; r < n_rec; r++) vtrace.push_back((double)info.input[5 * rec[r]]);
        }
        if (record && c == steps - 1)
            for (int64_t i = 0; i < 5 * n; i++) last[i] = (double)info.input[i];
    }
    clock_gettime(CLOCK_MONOTONIC, &t1);
    double secs = (t1.tv_sec - t0.tv_sec) + 1e-9 * (t1.tv_nsec - t0.tv_nsec);

    FILE *o = fopen(argv[2], "wb");
    if (!o) return 7;
    int64_t nrec_steps = (int64_t)raster_n.size();
    fwrite(&nrec_steps, 8, 1, o);
    fwrite(raster_n.data(), 8, raster_n.size(), o);
    int64_t nr = (int64_t)raster.size();
    fwrite(&nr, 8, 1, o);
    fwrite(raster.data(), 4, raster.size(), o);
    fwrite(vtrace.data(), 8, vtrace.size(), o);
    std::vector<int32_t> cnt(n);
    for (int64_t i = 0; i < n; i++) cnt[i] = neuron[i]->getFireCount();
    fwrite(cnt.data(), 4, n, o);
    fwrite(last.data(), 8, 5 * n, o);
    fwrite(&secs, 8, 1, o);
    fclose(o);
    printf("ref_driver: %lld neurons, %lld synapses, %lld cycles in %.6f s\n", (long long)n, (long long)s,
           (long long)steps, secs);
    return 0;
}
