"""Network descriptions shared by the tests and the benchmark harness.

A network is a dict of flat arrays in the reference's construction order:
  params   [n, 10] float64  LIFENeuron constructor arguments per neuron
                            (v_init, v_rest, v_reset, cm, tau_m, tau_refrac,
                             tau_syn_E, tau_syn_I, v_thresh, i_offset)
  pop_size [P]     int64    population sizes, global ids follow population order
  pop_tau  [P, 2]  float64  CompositeNeuron tau_syn_E / tau_syn_I of each population
  src, dst [S]     int32    synapses in creation (connect) order
  weight   [S]     float64  connect() weight, SI units (A)
  delay    [S]     float64  connect() delay in seconds
  type     [S]     uint8    SpikeType passed to connect (0 excitatory, 1 inhibitory)

write_net() serialises one for oracle/_ref/ref_driver_* (the reference's own
simulator built from its sources); the layout is the one ref_driver.cpp reads.
"""
import numpy as np


def lif_unit_net(which):
    """The four 3x10 LIF_brian nets of the reference's test/gpu/lif_unit{1..4}_test.cpp,
    whose v traces are the golden files test/lif_unit{1..4}_test_v.std."""
    N = 10
    base = [0.0, 0.0, 0.0, 1.0e-1, 50.0e-3, 0.0, 1.0, 1.0, 15.0e-3, 0.0]
    p0 = list(base); p0[9] = 100.0e-1
    p1 = list(base)
    p2 = list(base)
    if which == 4:
        p0[5] = 2e-4
        p1[5] = 1e-4
    params = np.array([p0] * N + [p1] * N + [p2] * N, dtype=np.float64)
    i = np.arange(N * N, dtype=np.float64)
    if which == 2:
        w0 = 1e-4 + i / (N * N) * 2e-3
        w1 = 2.1e-3 - i / (N * N) * 2e-3
    else:
        w0 = np.full(N * N, 1e-5)
        w1 = np.full(N * N, 2e-5)
    d0 = np.full(N * N, 2e-4 if which == 3 else 1e-4)
    d1 = np.full(N * N, 1e-4)
    k = np.arange(N * N)
    src = np.concatenate([k // N, N + k // N]).astype(np.int32)
    dst = np.concatenate([N + k % N, 2 * N + k % N]).astype(np.int32)
    return dict(params=params, pop_size=np.array([N, N, N], dtype=np.int64),
                pop_tau=np.ones((3, 2)), src=src, dst=dst,
                weight=np.concatenate([w0, w1]), delay=np.concatenate([d0, d1]),
                type=np.zeros(2 * N * N, dtype=np.uint8), dt=1.0e-4, steps=1000)


def write_net(path, net, steps, record_steps, rec_ids=None, dt=None):
    dt = net["dt"] if dt is None else dt
    rec_ids = np.zeros(0, np.int32) if rec_ids is None else np.asarray(rec_ids, np.int32)
    n = net["params"].shape[0]
    s = net["src"].shape[0]
    with open(path, "wb") as f:
        f.write(b"BSNT")
        np.array([n, s, steps, record_steps, len(net["pop_size"]), len(rec_ids)], np.int64).tofile(f)
        np.array([dt], np.float64).tofile(f)
        np.asarray(net["pop_size"], np.int64).tofile(f)
        np.asarray(net["pop_tau"], np.float64).tofile(f)
        np.asarray(net["params"], np.float64).tofile(f)
        np.asarray(net["src"], np.int32).tofile(f)
        np.asarray(net["dst"], np.int32).tofile(f)
        np.asarray(net["weight"], np.float64).tofile(f)
        np.asarray(net["delay"], np.float64).tofile(f)
        np.asarray(net["type"], np.uint8).tofile(f)
        rec_ids.tofile(f)


def syn_tau(net):
    """tau of each synapse as CompositeNeuron::createSynapse picks it
    (src/base/CompositeNeuron.h:61-79): the target population's tau_syn_E for
    excitatory connects, tau_syn_I for inhibitory ones."""
    pop_of = np.repeat(np.arange(len(net["pop_size"])), net["pop_size"])
    tp = pop_of[net["dst"]]
    return np.where(net["type"] == 0, net["pop_tau"][tp, 0], net["pop_tau"][tp, 1])
