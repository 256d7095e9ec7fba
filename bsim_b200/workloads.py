"""The CUBA LIF_brian workloads the engine is measured on, as generator specs.

Every network is the sparse random variant of the reference's standard_test
chain (test/gpu/standard_test.cpp:54-153): P populations of n LIF_brian neurons
(v_rest = v_reset = -65 mV, v_thresh = -50 mV, cm = 0.25 nF, tau_m = 20 ms,
tau_syn_E = 5 ms, tau_syn_I = 10 ms), chain k -> k+1 with p = 0.1, 20 % of the
populations with one extra remote projection, 80 % excitatory synapses with
weights U[0, w_max), inhibitory ones -U[0, 4 w_max), integer delays U{1..D}
steps, dt = 0.1 ms, i_offset U[0, i_max) per neuron and v_init U[-65, -50) mV.

The mean firing rate is set by i_offset (the recurrent input is balanced on
average). A 2 ms refractory period caps a LIF_brian neuron at 1/(20 steps) =
500 Hz, so the 500 Hz and 2 kHz presets shorten it (0.5 ms, 0.2 ms). The
i_max values were calibrated by simulation (mean rate over steps 1,000-2,000):
the presets on 10 x 1,000-neuron nets with the CPU oracle, and the large
configurations on the GPU at full size. In the 100-population chain the
recurrent inhibition silences a few populations (per-population rates span
0-1,280 Hz), so a larger i_offset raises the mean only slowly: i_max = 30 nA
gives ~430 Hz there.
"""
import numpy as np

from . import gen_spec

DT = 1.0e-4
W_MAX = 1.0e-10

# rate (Hz) -> (tau_refrac s, i_max A), calibrated on 10 x 1,000-neuron nets
RATE_PRESETS = {100: (2.0e-3, 3.2e-9), 500: (0.5e-3, 17.5e-9), 2000: (0.2e-3, 50.0e-9)}


def cuba(n_pop, pop_size, rate_hz=100, max_delay=6, seed=1, w_max=W_MAX, i_max=None):
    tref, imax = RATE_PRESETS[rate_hz]
    return gen_spec(seed=seed, n_pop=n_pop, pop_size=pop_size, max_delay=max_delay, w_max=w_max,
                    i_min=0.0, i_max=imax if i_max is None else i_max, tau_refrac=tref)


def standard_cpu(seed=1):
    """10 populations x 1,000 neurons, ~100 Hz, delays U{1..6}, 1 s (10,000 steps)."""
    return [cuba(10, 1000, 100, 6, seed)], 10000


def plain_1m(seed=1):
    """100 populations x 10,000 neurons (1e6 neurons, ~1.19e9 synapses), ~430 Hz (the 500 Hz
    preset's refractory period, i_max = 30 nA), delays U{1..6}, 1 s."""
    return [cuba(100, 10000, 500, 6, seed, i_max=30e-9)], 10000


def dense_1m(seed=1):
    """50 populations x 20,000 neurons (~2.36e9 synapses), ~2 kHz (i_max = 62.5 nA),
    delays U{1..50}, 0.5 s."""
    return [cuba(50, 20000, 2000, 50, seed, i_max=62.5e-9)], 5000


def batched(n_nets=256, seed=1):
    """n_nets independent networks of uneven size: populations U{5..40} x neurons
    U{500..8,000}, rate from {100, 500, 2000} Hz, delays U{1..6} or U{1..50}, 1 s."""
    rng = np.random.default_rng(seed)
    specs = []
    for k in range(n_nets):
        P = int(rng.integers(5, 41))
        n = int(rng.integers(500, 8001))
        rate = int(rng.choice([100, 500, 2000]))
        D = int(rng.choice([6, 50]))
        specs.append(cuba(P, n, rate, D, seed=int(rng.integers(1, 2**62))))
    return specs, 10000


def predicted_2m(seed=1):
    """200 populations x 10,000 neurons (2e6 neurons, ~2.4e9 synapses), delays U{1..20}, 2 s,
    i_offset U[0, 2.5 nA) under a 10 Hz square wave (x32, i.e. up to 80 nA, in the odd 50 ms
    half periods). Calibrated on the GPU at full size: ~5-15 Hz in the low half periods
    (drifting up slowly), ~800-1,000 Hz in the high ones."""
    sp = cuba(200, 10000, 500, 20, seed, i_max=2.5e-9)
    sp.drive_scale = 32.0
    sp.drive_half_period = 500
    return [sp], 20000


def scaled(spec, pop_size):
    """The same generator with smaller populations (scaled-down replica for CPU checks)."""
    s = cuba(spec.n_pop, pop_size, 100, spec.max_delay, spec.seed)
    for f, _ in type(spec)._fields_:
        if f != "pop_size":
            setattr(s, f, getattr(spec, f))
    return s
