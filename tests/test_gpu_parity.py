"""GPU parity: the CUDA engine, called through the C ABI, against the CPU oracle
on the same seeded networks.

Bars (fp32 dynamics):
  * ORDERED accumulation vs the oracle in reference order (= the reference's own
    simulator, see test_oracle.py): rasters, spike counts and state bit-identical.
  * EXACT accumulation vs the oracle in fixed-point mode with the engine's qexp:
    bit-identical; vs the reference order: raster identical for the first 1,000
    steps, v within 1e-5 relative, population rates within 1 %.
  * push vs pull, graph vs plain launches, batched vs alone, device-built vs
    host-built: bit-identical.
"""
import numpy as np
import pytest

import bsim_b200 as B
import netio
from bsim_b200 import workloads as W
from oracle import oracle

pytestmark = pytest.mark.gpu
DT = np.float32(1e-4)


def unit_arrays(which):
    net = netio.lif_unit_net(which)
    tau = netio.syn_tau(net).astype(np.float32)
    st, w = B.synapse_reset(net["delay"].astype(np.float32), net["weight"].astype(np.float32), tau, DT)
    return dict(params=net["params"].astype(np.float32), src=net["src"], dst=net["dst"], weight=w, delay_steps=st)


def engine_from(g, **opt):
    return B.Engine.from_arrays(g["params"], g["src"], g["dst"], g["weight"], g["delay_steps"], DT,
                                pop=g.get("pop"), instance=g.get("instance"), opts=B.options(**opt))


def run_checkpoints(eng, steps, every, cap=None):
    """Runs `steps` cycles recording the raster; returns (raster, [v at each checkpoint])."""
    n = eng.info().n_neurons
    eng.record(steps, cap or n * steps)
    vs = []
    done = 0
    while done < steps:
        k = min(every, steps - done)
        eng.run(k)
        done += k
        vs.append(eng.state()["v"])
    return eng.raster(), vs


def oracle_run(g, steps, mode, qexp=None, rec_ids=None):
    n = g["params"].shape[0]
    return oracle.run(g["params"], g["src"], g["dst"], g["weight"], g["delay_steps"], DT, steps,
                      record_steps=steps, rec_ids=np.arange(n) if rec_ids is None else rec_ids,
                      acc_mode=mode, qexp=qexp)


def same_raster(a, b, upto=None):
    upto = min(len(a), len(b)) if upto is None else upto
    for t in range(upto):
        if not np.array_equal(a[t], b[t]):
            return t
    return None


@pytest.mark.parametrize("which", [1, 2, 3, 4])
def test_unit_nets_ordered_bit_exact(which):
    g = unit_arrays(which)
    eng = engine_from(g, accumulate=B.ACC_ORDERED)
    raster, vs = run_checkpoints(eng, 1000, 100)
    ref = oracle_run(g, 1000, oracle.ACC_SEQUENTIAL)
    assert same_raster(raster, ref["raster"]) is None
    for k, v in enumerate(vs):
        assert np.array_equal(v, ref["v_trace"][100 * k + 99])
    gold = np.load(__file__.replace("test_gpu_parity.py", "golden/lif_unit_v.npz"))["unit%d" % which]
    for k, v in enumerate(vs):
        assert np.abs(v.astype(np.float64) - gold[100 * k + 99]).max() < 3.5e-7
    assert np.array_equal(eng.fire_count(), ref["fire_count"])


@pytest.mark.parametrize("which", [1, 2, 3, 4])
@pytest.mark.parametrize("delivery", [B.DELIVERY_PUSH, B.DELIVERY_PULL])
def test_unit_nets_exact_bit_exact(which, delivery):
    g = unit_arrays(which)
    eng = engine_from(g, delivery=delivery)
    raster, vs = run_checkpoints(eng, 1000, 250)
    ref = oracle_run(g, 1000, oracle.ACC_FIXED, qexp=int(eng.qexp()[0]))
    assert same_raster(raster, ref["raster"]) is None
    for k, v in enumerate(vs):
        assert np.array_equal(v, ref["v_trace"][250 * k + 249])


@pytest.fixture(scope="module")
def c0():
    specs, _ = W.standard_cpu(seed=1)
    g = B.gen_host(specs[0])
    return specs[0], g


def test_device_builder_matches_host_builder(c0):
    spec, g = c0
    a = B.Engine.generated(spec, DT)
    b = engine_from(g)
    assert a.info().n_synapses == len(g["src"])
    assert np.array_equal(a.qexp(), b.qexp())
    ra, _ = run_checkpoints(a, 300, 300)
    rb, _ = run_checkpoints(b, 300, 300)
    assert same_raster(ra, rb) is None
    sa, sb = a.state(), b.state()
    for k in sa:
        assert np.array_equal(sa[k], sb[k])
    assert a.info().events_total == b.info().events_total


def test_c0_exact_push_vs_oracle(c0):
    """1,000 steps of the 10 x 1,000 CUBA net: bit-exact against the fixed-point
    oracle; against the reference order: identical raster, v within 1e-5 relative."""
    spec, g = c0
    eng = B.Engine.generated(spec, DT)
    raster, vs = run_checkpoints(eng, 1000, 500)
    q = int(eng.qexp()[0])
    fx = oracle_run(g, 1000, oracle.ACC_FIXED, qexp=q)
    assert same_raster(raster, fx["raster"]) is None
    assert np.array_equal(vs[-1], fx["v_trace"][-1])
    assert np.array_equal(eng.fire_count(), fx["fire_count"])
    assert eng.info().events_total == fx["events_per_step"].sum()
    sq = oracle_run(g, 1000, oracle.ACC_SEQUENTIAL)
    assert same_raster(raster, sq["raster"]) is None
    v_ref = sq["v_trace"][-1].astype(np.float64)
    assert np.all(np.abs(vs[-1] - v_ref) <= 1e-5 * np.abs(v_ref))


def test_c0_ordered_pull_bit_exact_vs_reference_order(c0):
    spec, g = c0
    eng = B.Engine.generated(spec, DT, opts=B.options(accumulate=B.ACC_ORDERED))
    raster, vs = run_checkpoints(eng, 2000, 1000)
    sq = oracle_run(g, 2000, oracle.ACC_SEQUENTIAL)
    assert same_raster(raster, sq["raster"]) is None
    assert np.array_equal(vs[-1], sq["v_trace"][-1])
    assert np.array_equal(eng.fire_count(), sq["fire_count"])


def test_c0_full_second_rates_within_1pct(c0):
    """The whole 1 s (10,000 steps): per-population rates of the EXACT engine
    within 1 % of the reference order."""
    spec, g = c0
    eng = B.Engine.generated(spec, DT)
    eng.run(10000)
    sq = oracle_run(g, 10000, oracle.ACC_SEQUENTIAL, rec_ids=np.zeros(0, np.int32))
    ra = eng.fire_count().reshape(spec.n_pop, -1).sum(1)
    rb = sq["fire_count"].reshape(spec.n_pop, -1).sum(1)
    assert np.all(np.abs(ra - rb) <= 0.01 * rb)


def test_push_pull_graph_identical(c0):
    spec, _ = c0
    outs = []
    for opt in (dict(), dict(delivery=B.DELIVERY_PULL), dict(graph_steps=0), dict(graph_steps=7, block_threads=128)):
        eng = B.Engine.generated(spec, DT, opts=B.options(**opt))
        r, vs = run_checkpoints(eng, 500, 500)
        outs.append((r, vs[-1], eng.fire_count(), eng.info().events_total))
    for o in outs[1:]:
        assert same_raster(outs[0][0], o[0]) is None
        assert np.array_equal(outs[0][1], o[1]) and np.array_equal(outs[0][2], o[2]) and outs[0][3] == o[3]


def test_batched_equals_alone():
    """Three uneven networks (different rates and delay ranges) packed into one
    engine give each network's own raster and state bit for bit."""
    specs = [W.cuba(5, 700, 100, 6, seed=21), W.cuba(7, 500, 500, 50, seed=22), W.cuba(6, 600, 2000, 6, seed=23)]
    both = B.Engine.generated(specs, DT)
    rb, _ = run_checkpoints(both, 400, 400)
    sb = both.state()
    base = 0
    for sp in specs:
        n = sp.n_pop * sp.pop_size
        alone = B.Engine.generated(sp, DT)
        ra, _ = run_checkpoints(alone, 400, 400)
        sa = alone.state()
        for t in range(400):
            mine = rb[t][(rb[t] >= base) & (rb[t] < base + n)] - base
            assert np.array_equal(mine, ra[t]), t
        assert np.array_equal(sb["v"][base:base + n], sa["v"])
        base += n


@pytest.mark.parametrize("name,spec,steps", [
    ("dense_scaled", W.cuba(50, 400, 2000, 50, seed=3), 300),
    ("plain_scaled", W.cuba(100, 200, 500, 6, seed=4), 300),
])
def test_scaled_replicas_vs_oracle(name, spec, steps):
    """Scaled-down replicas of the 1e6-neuron configurations (same generator,
    smaller populations): bit-exact against the fixed-point oracle."""
    g = B.gen_host(spec)
    eng = B.Engine.generated(spec, DT)
    raster, vs = run_checkpoints(eng, steps, steps)
    fx = oracle_run(g, steps, oracle.ACC_FIXED, qexp=int(eng.qexp()[0]))
    assert same_raster(raster, fx["raster"]) is None
    assert np.array_equal(vs[-1], fx["v_trace"][-1])
    assert eng.info().events_total == fx["events_per_step"].sum()


@pytest.mark.parametrize("opts", [dict(), dict(tile_size=300), dict(tile_size=256, block_threads=256)])
def test_tiled_delivery_identical_to_push(c0, opts):
    """Target-tiled delivery (shared-memory sums) equals push delivery bit for bit,
    device-built and host-built, including tiles that straddle populations."""
    spec, g = c0
    ref = B.Engine.generated(spec, DT)
    r_ref, v_ref = run_checkpoints(ref, 400, 400)
    for eng in (B.Engine.generated(spec, DT, opts=B.options(delivery=B.DELIVERY_TILE, **opts)),
                engine_from(g, delivery=B.DELIVERY_TILE, **opts)):
        r, v = run_checkpoints(eng, 400, 400)
        assert same_raster(r, r_ref) is None
        assert np.array_equal(v[-1], v_ref[-1])
        assert eng.info().events_total == ref.info().events_total


def test_tiled_batched_long_delays_equal_alone():
    specs = [W.cuba(6, 700, 2000, 50, seed=41), W.cuba(5, 900, 100, 6, seed=42)]
    both = B.Engine.generated(specs, DT, opts=B.options(delivery=B.DELIVERY_TILE, tile_size=512))
    rb, _ = run_checkpoints(both, 300, 300)
    base = 0
    for sp in specs:
        n = sp.n_pop * sp.pop_size
        alone = B.Engine.generated(sp, DT)
        ra, _ = run_checkpoints(alone, 300, 300)
        for t in range(300):
            mine = rb[t][(rb[t] >= base) & (rb[t] < base + n)] - base
            assert np.array_equal(mine, ra[t]), t
        base += n


def test_square_wave_drive_vs_oracle():
    """Square-wave drive (i_offset x drive_scale in odd half periods): device-built
    and host-built (bsim_set_drive) engines both bit-exact against the oracle."""
    spec = W.cuba(6, 500, 100, 6, seed=51)
    spec.i_max = 1.0e-9
    spec.drive_scale = 20.0
    spec.drive_half_period = 60
    g = B.gen_host(spec)
    hi = g["params"].copy()
    hi[:, 9] = (g["params"][:, 9] * np.float32(20.0)).astype(np.float32)
    dev = B.Engine.generated(spec, DT)
    host = engine_from(g)
    host.set_drive(hi, 60)
    rd, vd = run_checkpoints(dev, 300, 300)
    rh, vh = run_checkpoints(host, 300, 300)
    fx = oracle.run(g["params"], g["src"], g["dst"], g["weight"], g["delay_steps"], DT, 300, record_steps=300,
                    rec_ids=np.arange(g["params"].shape[0]), acc_mode=oracle.ACC_FIXED,
                    qexp=int(dev.qexp()[0]), params_alt=hi, half_period=60)
    assert same_raster(rd, fx["raster"]) is None and same_raster(rh, fx["raster"]) is None
    assert np.array_equal(vd[-1], fx["v_trace"][-1]) and np.array_equal(vh[-1], fx["v_trace"][-1])
    lo_rate = sum(len(r) for r in fx["raster"][:60]) / 60
    hi_rate = sum(len(r) for r in fx["raster"][60:120]) / 60
    assert hi_rate > 3 * lo_rate


# ---------------------------------------------------------------------------
# Tiled and AUTO delivery (the benchmark's default modes) against the oracle at
# the shapes the benchmark runs: scaled replicas of the 1e6-neuron (100
# populations, delays 1-6), dense (50 populations, delays 1-50) and
# predictor-scheduled (200 populations, delays 1-20, square-wave drive)
# configurations, with the automatic tile size (many parts per tile, so most
# blocks help), tiles straddling populations with ~3 parts each, and one tile
# for the whole network (every block but one helps). Reference semantics:
# update_dense_static_hit, src/synapse/static/static.cu:59-96.
# ---------------------------------------------------------------------------
_FIXED = {}


def replica(name):
    if name == "plain":
        return W.scaled(W.plain_1m(1)[0][0], 200)
    if name == "dense":
        return W.scaled(W.dense_1m(1)[0][0], 400)
    if name == "square":
        return W.scaled(W.predicted_2m(1)[0][0], 100)
    raise KeyError(name)


def fixed_reference(name, steps, qexp):
    """The fixed-point oracle's run of a replica (cached per test session)."""
    key = (name, steps, qexp)
    if key not in _FIXED:
        spec = replica(name)
        g = B.gen_host(spec)
        kw = {}
        if spec.drive_half_period > 0:
            hi = g["params"].copy()
            hi[:, 9] = (g["params"][:, 9] * np.float32(spec.drive_scale)).astype(np.float32)
            kw = dict(params_alt=hi, half_period=int(spec.drive_half_period))
        _FIXED[key] = (g, oracle.run(g["params"], g["src"], g["dst"], g["weight"], g["delay_steps"], DT, steps,
                                     record_steps=steps, rec_ids=np.arange(g["params"].shape[0]),
                                     acc_mode=oracle.ACC_FIXED, qexp=qexp, **kw))
    return _FIXED[key]


def check_vs_fixed(eng, name, steps):
    raster, vs = run_checkpoints(eng, steps, steps)
    g, fx = fixed_reference(name, steps, int(eng.qexp()[0]))
    assert sum(len(r) for r in raster) > 0
    assert same_raster(raster, fx["raster"]) is None
    assert np.array_equal(vs[-1], fx["v_trace"][-1])
    assert np.array_equal(eng.fire_count(), fx["fire_count"])
    assert eng.info().events_total == fx["events_per_step"].sum()


@pytest.mark.parametrize("name,opts", [
    ("plain", dict()),
    ("plain", dict(tile_size=150)),
    ("plain", dict(tile_size=20000)),
    ("dense", dict()),
    ("square", dict()),
])
def test_tiled_delivery_vs_oracle_at_bench_shapes(name, opts):
    eng = B.Engine.generated(replica(name), DT, opts=B.options(delivery=B.DELIVERY_TILE, **opts))
    check_vs_fixed(eng, name, 1000)


def test_auto_delivery_vs_oracle_switching_modes():
    """AUTO delivery under the firing predictor, with cost models whose crossover
    sits inside the network's range of activity, so that cycles go both ways:
    still bit-identical to the oracle."""
    spec = replica("plain")
    eng = B.Engine.generated(spec, DT, opts=B.options(delivery=B.DELIVERY_AUTO))
    eng.enable_pop_stats(64)
    g, fx = fixed_reference("plain", 1000, int(eng.qexp()[0]))
    work = np.median(fx["events_per_step"][100:])
    eng.set_predictor(B.mlp_init(5), tolerance=0.25, cost_push=[0.0, 1.0], cost_tile=[float(work), 0.0])
    check_vs_fixed(eng, "plain", 1000)
    st = eng.predictor_stats()
    assert 0 < st.tile_cycles < st.cycles


def test_tiled_delivery_rates_over_a_full_second():
    """10,000 cycles (1 s) of the 1e6-neuron configuration's replica with tiled
    delivery: per-population rates within 1 % of the reference order."""
    spec = replica("plain")
    g = B.gen_host(spec)
    eng = B.Engine.generated(spec, DT, opts=B.options(delivery=B.DELIVERY_TILE))
    eng.run(10000)
    sq = oracle_run(g, 10000, oracle.ACC_SEQUENTIAL, rec_ids=np.zeros(0, np.int32))
    ra = eng.fire_count().reshape(spec.n_pop, -1).sum(1).astype(np.float64)
    rb = sq["fire_count"].reshape(spec.n_pop, -1).sum(1).astype(np.float64)
    assert rb.sum() > 0
    assert np.all(np.abs(ra - rb) <= 0.01 * np.maximum(rb, 100))
