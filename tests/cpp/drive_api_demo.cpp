// A user program of the reference's C++ API with input-drive neurons, compiled
// against bsim_b200's include/BSim.h: a Constant_spikes and a Poisson_spikes
// population drive one LIF_brian population through all-to-all connections
// (the pattern of the reference's test/gpu/gpusim_unit_test.cpp), 0.2 s with SGSim.
#include <stdlib.h>

#include "BSim.h"

int main()
{
    const int NC = 4, NP = 6, NL = 8;
    Network net;
    Population<Constant_spikes> *c =
        net.createPopulation(0, NC, Constant_spikes(ConstantNeuron(0.02, 0.0, 0.15), 1e-3, 1e-3));
    Population<Poisson_spikes> *p =
        net.createPopulation(1, NP, Poisson_spikes(PoissonNeuron(40.0, 1e-3, 0.005, 1000.0), 1e-3, 1e-3));
    Population<LIF_brian> *l = net.createPopulation(
        2, NL, LIF_brian(LIFENeuron(-0.065, -0.065, -0.065, 0.25e-9, 20e-3, 2e-3, 5e-3, 10e-3, -0.050, 0.1e-9),
                         5e-3, 10e-3));
    real *wc = new real[NC * NL], *wp = new real[NP * NL];
    for (int i = 0; i < NC * NL; i++) wc[i] = 1e-9 + 1e-10 * (i % 7);
    for (int i = 0; i < NP * NL; i++) wp[i] = 2e-9 - 1e-10 * (i % 5);
    real *dc = getConstArray((real)2e-4, NC * NL);
    real *dp = getConstArray((real)5e-4, NP * NL);
    net.connect(c, l, wc, dc, NULL, NC * NL);
    net.connect(p, l, wp, dp, NULL, NP * NL);
    SGSim sg(&net, 1.0e-4);
    int rc = sg.run(0.2);
    printf("drive_api_demo: rc=%d\n", rc);
    return rc == 0 ? 0 : 1;
}
