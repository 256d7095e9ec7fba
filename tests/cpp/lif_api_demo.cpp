// A user program of the reference's C++ API, compiled against bsim_b200's
// include/BSim.h: three 10-neuron LIF_brian populations chained all-to-all
// (the shape of the reference's test/gpu/lif_unit{1..4}_test.cpp), simulated
// for 0.1 s with SGSim. argv[1] picks the variant 1..4.
#include <stdlib.h>

#include "BSim.h"

int main(int argc, char **argv)
{
    const int which = argc > 1 ? atoi(argv[1]) : 1;
    const int N = 10;
    Network net;
    real ref0 = which == 4 ? 2e-4 : 0.0, ref1 = which == 4 ? 1e-4 : 0.0;
    Population<LIF_brian> *a = net.createPopulation(
        N, LIF_brian(LIFENeuron(0.0, 0.0, 0.0, 1.0e-1, 50.0e-3, ref0, 1.0, 1.0, 15.0e-3, 100.0e-1), 1.0, 1.0));
    Population<LIF_brian> *b = net.createPopulation(
        N, LIF_brian(LIFENeuron(0.0, 0.0, 0.0, 1.0e-1, 50.0e-3, ref1, 1.0, 1.0, 15.0e-3, 0.0e-3), 1.0, 1.0));
    Population<LIF_brian> *c = net.createPopulation(
        N, LIF_brian(LIFENeuron(0.0, 0.0, 0.0, 1.0e-1, 50.0e-3, 0.0, 1.0, 1.0, 15.0e-3, 0.0e-3), 1.0, 1.0));
    real *w0, *w1;
    if (which == 2) {
        w0 = new real[N * N];
        w1 = new real[N * N];
        for (int i = 0; i < N * N; i++) {
            w0[i] = 1e-4 + (double)i / (double)(N * N) * 2e-3;
            w1[i] = 2.1e-3 - (double)i / (double)(N * N) * 2e-3;
        }
    } else {
        w0 = getConstArray((real)1e-5, N * N);
        w1 = getConstArray((real)2e-5, N * N);
    }
    real *d0 = getConstArray((real)(which == 3 ? 2e-4 : 1e-4), N * N);
    real *d1 = getConstArray((real)1e-4, N * N);
    net.connect(a, b, w0, d0, NULL, N * N);
    net.connect(b, c, w1, d1, NULL, N * N);
    SGSim sg(&net, 1.0e-4);
    int rc = sg.run(0.1);
    printf("lif_api_demo %d: rc=%d\n", which, rc);
    return rc == 0 ? 0 : 1;
}
