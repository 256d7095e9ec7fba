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


def drive_net(seed=1, lif_size=200):
    """A network with input-drive neurons (kind 2 Poisson_spikes, kind 1 Constant_spikes)
    feeding two LIF_brian populations, in float32 engine form (dt = 0.1 ms).

    Population 0: 70 Poisson neurons, rates 3.5 .. 20000.5 cycles (every level of the
      sampler), refract 0 / 0.5 ms, start 0 / 10 ms, durations 1000 s or 0.2 s.
    Population 1: 20 Constant neurons, fire_rate 0.4 / 0.05 / 1.0 / 0.013 per cycle,
      start 5 ms, end 150 ms or 1e9 s (clamped).
    Populations 2, 3: LIF_brian, subthreshold i_offset; 0 -> 2, 1 -> 3, 2 -> 3 (E),
      3 -> 2 (I), and 2 -> 0 (input that drive neurons ignore). Delays U{1..8} steps.
    Returns params [n, 10], kind [n], pop [n], src, dst, weight, delay_steps."""
    rng = np.random.default_rng(seed)
    rates = np.repeat([3.5, 20.0, 70.25, 300.0, 1500.0, 6000.0, 20000.5], 10).astype(np.float32)
    nP, nC, nL = rates.size, 20, lif_size
    n = nP + nC + 2 * nL
    params = np.zeros((n, 10), np.float32)
    kind = np.zeros(n, np.uint8)
    pop = np.repeat(np.arange(4, dtype=np.int32), [nP, nC, nL, nL])
    i = np.arange(nP)
    kind[:nP] = 2
    params[:nP, 0] = rates
    params[:nP, 1] = np.where(i % 2 == 0, 0.0, 5e-4)
    params[:nP, 2] = np.where((i // 2) % 2 == 0, 0.0, 1e-2)
    params[:nP, 3] = np.where(i % 5 == 4, 0.2, 1000.0)
    c = np.arange(nC)
    kind[nP:nP + nC] = 1
    params[nP:nP + nC, 0] = np.array([0.4, 0.05, 1.0, 0.013], np.float32)[c % 4]
    params[nP:nP + nC, 1] = 5e-3
    params[nP:nP + nC, 2] = np.where(c < nC // 2, 0.15, 1e9)
    lif = [-0.065, -0.065, -0.065, 0.25e-9, 20e-3, 2e-3, 5e-3, 10e-3, -0.050, 0.0]
    params[nP + nC:] = lif
    params[nP + nC:, 0] = rng.uniform(-0.065, -0.055, 2 * nL)
    params[nP + nC:, 9] = rng.uniform(0.0, 0.15e-9, 2 * nL)
    base = [0, nP, nP + nC, nP + nC + nL]
    size = [nP, nC, nL, nL]
    src, dst, w = [], [], []
    for a, b, p, lo, hi in [(0, 2, 0.2, 0.0, 2e-9), (1, 3, 0.5, 0.0, 3e-10), (2, 3, 0.1, 0.0, 2e-10),
                            (3, 2, 0.1, -4e-10, 0.0), (2, 0, 0.05, 0.0, 1e-10)]:
        m = rng.random((size[a], size[b])) < p
        s_, d_ = np.nonzero(m)
        src.append(s_ + base[a])
        dst.append(d_ + base[b])
        w.append(rng.uniform(lo, hi, s_.size))
    src = np.concatenate(src).astype(np.int32)
    dst = np.concatenate(dst).astype(np.int32)
    weight = np.concatenate(w).astype(np.float32)
    delay = rng.integers(1, 9, src.size).astype(np.int32)
    return dict(params=params, kind=kind, pop=pop, src=src, dst=dst, weight=weight, delay_steps=delay)
