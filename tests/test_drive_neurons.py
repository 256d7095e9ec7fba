"""Input-drive neurons (Constant_spikes, Poisson_spikes) stepped with the LIF
neurons. CPU tests pin the oracle to the reference's GPU kernel rules
(src/neuron/constant/constant.cu:18-22, src/neuron/poisson/poisson.cu:9-31) and
check the reproducible Poisson sampler's distribution; GPU tests compare the
engine with the oracle bit for bit on a mixed network."""
import ctypes

import numpy as np
import pytest

import bsim_b200 as B
import netio
from oracle import oracle

DT = np.float32(1e-4)


def drive_only(params, kind, steps, seed=0):
    """Oracle run of drive neurons without synapses: their spike cycles."""
    n = params.shape[0]
    r = oracle.run(params, np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32),
                   np.zeros(0, np.int32), DT, steps, record_steps=steps, kind=kind, input_seed=seed)
    cycles = [[] for _ in range(n)]
    for t, ids in enumerate(r["raster"]):
        for j in ids:
            cycles[j].append(t)
    return cycles, r


def test_constant_neuron_follows_reference_gpu_rule():
    """update_constant_neuron: fires at t iff t < end_cycle and
    (t - start_cycle) * fire_rate > fire_count, in fp32; cycles = (int)(time / dt)."""
    rates = np.array([0.4, 0.05, 1.0, 0.013, 0.0, 0.37], np.float32)
    starts = np.array([0.0, 5e-4, 1e-3, 0.0, 0.0, 2.3e-3], np.float32)
    ends = np.array([2e-3, 1e9, 0.05, 1e9, 1e9, 0.0311], np.float32)
    n = rates.size
    params = np.zeros((n, 10), np.float32)
    params[:, 0], params[:, 1], params[:, 2] = rates, starts, ends
    steps = 600
    got, _ = drive_only(params, np.ones(n, np.uint8), steps)
    for j in range(n):
        sc = int(np.float32(starts[j]) / DT)
        q = np.float32(ends[j]) / DT
        ec = 2**31 - 1 if q >= np.float32(2**31) else int(q)
        want, cnt = [], 0
        for t in range(steps):
            if t < ec and np.float32(t - sc) * rates[j] > np.float32(cnt):
                want.append(t)
                cnt += 1
        assert got[j] == want, j
    # rate 0.4 from cycle 0: the first spikes of the rule written out
    assert got[0][:5] == [1, 3, 6, 8, 11]


def test_poisson_neuron_follows_reference_gpu_rule():
    """update_poisson_neuron / reset_poisson_neuron: the first spike at
    (int)(start/dt) + Poisson(rate), then gaps of 1 + Poisson(rate) + refrac_step,
    no spike after end_cycle; over many neurons the mean gap is 1 + rate + refrac_step."""
    n = 400
    params = np.zeros((n, 10), np.float32)
    params[:, 0] = 30.0
    params[:, 1] = np.where(np.arange(n) < n // 2, 0.0, 1e-3)  # refract: 0 or 10 steps
    params[:, 2] = 2e-3  # start: cycle 20
    params[:, 3] = 0.3   # duration: end cycle 3020
    steps = 4000
    got, _ = drive_only(params, np.full(n, 2, np.uint8), steps, seed=11)
    gaps = {0: [], 10: []}
    for j in range(n):
        c = np.array(got[j])
        rs = 0 if j < n // 2 else 10
        assert c[0] >= 20 and c[-1] <= 3020
        g = np.diff(c)
        assert np.all(g >= 1 + rs)
        gaps[rs] += list(g)
    for rs, g in gaps.items():
        g = np.asarray(g, np.float64)
        want = 1 + 30.0 + rs
        assert abs(g.mean() - want) < 4 * np.sqrt(30.0 / g.size), (rs, g.mean())
        assert abs(g.var() / 30.0 - 1) < 0.05


@pytest.mark.parametrize("rate", [0.7, 3.5, 40.0, 100.0])
def test_poisson_sampler_matches_pmf(rate):
    """Chi-square goodness of fit of 200,000 draws against the Poisson pmf."""
    from scipy import stats
    d = oracle.poisson_draws(3, rate, 200000)
    k = np.arange(0, int(rate + 8 * np.sqrt(rate) + 10))
    pmf = stats.poisson.pmf(k, rate)
    obs = np.bincount(np.minimum(d, k[-1]), minlength=k.size)[:k.size].astype(np.float64)
    exp = pmf * d.size
    exp[-1] += d.size * stats.poisson.sf(k[-1], rate)
    keep = exp > 5
    chi2 = ((obs[keep] - exp[keep]) ** 2 / exp[keep]).sum() + 0.0
    dof = keep.sum() - 1
    assert stats.chi2.sf(chi2, dof) > 1e-4


@pytest.mark.parametrize("rate", [64.0, 700.25, 5000.0, 20000.5, 100000.0])
def test_poisson_sampler_moments_large_rates(rate):
    """The table levels: mean and variance of 100,000 draws within 5 standard errors."""
    d = oracle.poisson_draws(17, rate, 100000).astype(np.float64)
    se_mean = np.sqrt(rate / d.size)
    se_var = rate * np.sqrt(2.0 / d.size)
    assert abs(d.mean() - rate) < 5 * se_mean
    assert abs(d.var() - rate) < 5 * se_var


def test_create_mixed_rejects_bad_kinds_and_rates():
    """Argument errors come back as BSIM_ERR_ARG before any device work."""
    L = B.lib()
    params = np.zeros((2, 10), np.float32)
    params[:, 0] = 5.0
    z32 = np.zeros(0, np.int32)
    opts = B.options()
    h = ctypes.c_void_p()
    for kind, rate in [([0, 7], 5.0), ([2, 2], -1.0), ([2, 2], 2.0**25), ([2, 2], float("nan"))]:
        params[:, 0] = rate
        k = np.array(kind, np.uint8)
        rc = L.bsim_create_mixed(params.ctypes.data, k.ctypes.data, 2, None, None, z32.ctypes.data,
                                 z32.ctypes.data, None, z32.ctypes.data, 0, DT, 1, ctypes.byref(opts),
                                 ctypes.byref(h))
        assert rc == -1  # BSIM_ERR_ARG


# ---------------------------------------------------------------------------
# GPU parity
# ---------------------------------------------------------------------------
def engine(g, seed, **opt):
    return B.Engine.from_arrays(g["params"], g["src"], g["dst"], g["weight"], g["delay_steps"], DT,
                                pop=g["pop"], instance=g.get("instance"), kind=g["kind"], input_seed=seed,
                                opts=B.options(**opt))


def run_engine(eng, steps, cap):
    eng.record(steps, cap)
    eng.run(steps)
    return eng.raster()


def first_diff(a, b):
    for t in range(min(len(a), len(b))):
        if not np.array_equal(a[t], b[t]):
            return t
    return None


def drive_state_ints(st, n):
    """The engine's state slots of drive neurons as the oracle's final_state holds them."""
    out = np.zeros((n, 3), np.int64)
    out[:, 0] = st["i_E"].view(np.int32)
    out[:, 1] = st["i_I"].view(np.int32)
    out[:, 2] = st["refrac"]
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("delivery", [B.DELIVERY_PUSH, B.DELIVERY_PULL])
def test_mixed_network_exact_vs_oracle(delivery):
    """25,000 cycles (Poisson rates up to 20,000 cycles reach every sampler level on
    the device): raster, spike counts and drive-neuron counters bit-identical to the
    fixed-point oracle."""
    g = netio.drive_net(1)
    n = g["params"].shape[0]
    steps = 25000
    eng = engine(g, 5, delivery=delivery)
    q = int(eng.qexp()[0])
    ras = run_engine(eng, steps, 600000)
    ref = oracle.run(g["params"], g["src"], g["dst"], g["weight"], g["delay_steps"], DT, steps,
                     record_steps=steps, acc_mode=oracle.ACC_FIXED, qexp=q, kind=g["kind"], input_seed=5,
                     raster_cap=600000)
    assert first_diff(ras, ref["raster"]) is None
    assert np.array_equal(eng.fire_count(), ref["fire_count"])
    st = eng.state()
    drv = g["kind"] != 0
    # the oracle keeps these counters as fp32 values (INT32_MAX rounds to 2^31 there too)
    assert np.array_equal(drive_state_ints(st, n)[drv].astype(np.float32), ref["final_state"][drv, 1:])
    lif = ~drv
    assert np.array_equal(st["v"][lif], ref["final_state"][lif, 0])
    assert eng.info().events_total == ref["events_per_step"].sum()


@pytest.mark.gpu
def test_mixed_network_ordered_vs_reference_order():
    """ORDERED accumulation: bit-identical to the oracle's reference-order sums."""
    g = netio.drive_net(2)
    steps = 3000
    eng = engine(g, 9, accumulate=B.ACC_ORDERED)
    ras = run_engine(eng, steps, 200000)
    ref = oracle.run(g["params"], g["src"], g["dst"], g["weight"], g["delay_steps"], DT, steps,
                     record_steps=steps, acc_mode=oracle.ACC_SEQUENTIAL, kind=g["kind"], input_seed=9,
                     raster_cap=200000)
    assert first_diff(ras, ref["raster"]) is None
    lif = g["kind"] == 0
    assert np.array_equal(eng.state()["v"][lif], ref["final_state"][lif, 0])


@pytest.mark.gpu
def test_mixed_networks_batched_equal_alone():
    """Two mixed networks packed in one engine: each one's spikes equal its run alone
    (Poisson draws are keyed by the neuron's id within its own network)."""
    a, b = netio.drive_net(3, lif_size=150), netio.drive_net(4, lif_size=250)
    na = a["params"].shape[0]
    both = {k: np.concatenate([a[k], b[k]]) for k in ("params", "kind")}
    both["pop"] = np.concatenate([a["pop"], b["pop"] + 4])
    both["instance"] = np.repeat(np.array([0, 1], np.int32), [na, b["params"].shape[0]])
    both["src"] = np.concatenate([a["src"], b["src"] + na])
    both["dst"] = np.concatenate([a["dst"], b["dst"] + na])
    both["weight"] = np.concatenate([a["weight"], b["weight"]])
    both["delay_steps"] = np.concatenate([a["delay_steps"], b["delay_steps"]])
    steps = 2000
    rb = run_engine(engine(both, 21), steps, 400000)
    for net, lo in ((a, 0), (b, na)):
        hi = lo + net["params"].shape[0]
        ra = run_engine(engine(net, 21), steps, 400000)
        for t in range(steps):
            mine = rb[t][(rb[t] >= lo) & (rb[t] < hi)] - lo
            assert np.array_equal(mine, ra[t]), t
