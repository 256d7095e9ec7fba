"""Edge cases of the step against the oracle (EXACT accumulation, every delivery
mode that applies): no synapses, a single neuron and ragged sizes, the maximum
delay, every neuron firing every cycle (full fire-ring slots), sources without
out-synapses and targets without in-synapses."""
import numpy as np
import pytest

import bsim_b200 as B
from oracle import oracle

pytestmark = pytest.mark.gpu
DT = np.float32(1e-4)
LIF = [-0.065, -0.065, -0.065, 0.25e-9, 20e-3, 2e-3, 5e-3, 10e-3, -0.050, 0.0]


def lif_params(n, i_offset, refract=2e-3, seed=0):
    rng = np.random.default_rng(seed)
    p = np.tile(np.array(LIF, np.float32), (n, 1))
    p[:, 0] = rng.uniform(-0.065, -0.051, n)
    p[:, 5] = refract
    p[:, 9] = i_offset if np.isscalar(i_offset) else np.asarray(i_offset, np.float32)
    return p


def check(params, src, dst, w, d, steps, modes=("push", "pull", "tile"), cap=None):
    """Runs the network in each delivery mode and compares raster, spike counts,
    membrane potentials and delivered events with the fixed-point oracle."""
    n = params.shape[0]
    src, dst = np.asarray(src, np.int32), np.asarray(dst, np.int32)
    w, d = np.asarray(w, np.float32), np.asarray(d, np.int32)
    opts = {"push": dict(), "pull": dict(delivery=B.DELIVERY_PULL), "tile": dict(delivery=B.DELIVERY_TILE)}
    cap = cap or max(n * steps, 1)
    ref = None
    for m in modes:
        eng = B.Engine.from_arrays(params, src, dst, w, d, DT, opts=B.options(**opts[m]))
        eng.record(steps, cap)
        eng.run(steps)
        ras = eng.raster()
        if ref is None:
            q = int(eng.qexp()[0])
            ref = oracle.run(params, src, dst, w, d, DT, steps, record_steps=steps, acc_mode=oracle.ACC_FIXED,
                             qexp=q, raster_cap=cap)
        assert len(ras) == steps
        for t in range(steps):
            assert np.array_equal(ras[t], ref["raster"][t]), (m, t)
        assert np.array_equal(eng.fire_count(), ref["fire_count"]), m
        assert np.array_equal(eng.state()["v"], ref["final_state"][:, 0]), m
        assert eng.info().events_total == ref["events_per_step"].sum(), m
        eng.close()
    return ref


def test_no_synapses():
    r = check(lif_params(100, np.linspace(0.0, 0.5e-9, 100)), [], [], [], [], 600)
    assert r["fire_count"].sum() > 0 and r["events_per_step"].sum() == 0


@pytest.mark.parametrize("n", [1, 31, 33, 1007])
def test_ragged_sizes(n):
    rng = np.random.default_rng(n)
    params = lif_params(n, rng.uniform(0.1e-9, 0.4e-9, n), seed=n)
    s = 4 * n
    src, dst = rng.integers(0, n, s), rng.integers(0, n, s)
    w = rng.uniform(-2e-10, 3e-10, s)
    d = rng.integers(1, 7, s)
    check(params, src, dst, w, d, 400)


def test_max_delay():
    """A spike fired at cycle t arrives through a delay of BSIM_MAX_DELAY steps (push only:
    pull takes delays up to 256 and the tiled copy up to 64)."""
    params = lif_params(3, [0.4e-9, 0.0, 0.0], refract=0.05)
    d = B.MAX_DELAY
    r = check(params, [0, 0], [1, 2], [5e-8, 5e-8], [d, 3], d + 200, modes=("push",))
    fired0 = [t for t, ids in enumerate(r["raster"]) if 0 in ids]
    fired1 = [t for t, ids in enumerate(r["raster"]) if 1 in ids]
    # delivered in the synapse phase of t + d, added to i_E by the update of t + d + 1,
    # seen by v in the update of t + d + 2 (as for the 3-step synapse into neuron 2)
    fired2 = [t for t, ids in enumerate(r["raster"]) if 2 in ids]
    assert fired0 and fired1 and fired1[0] == fired0[0] + d + 2 and fired2[0] == fired0[0] + 3 + 2


def test_every_neuron_fires_every_cycle():
    """No refractory period and a suprathreshold drive: all N ids in every ring slot,
    all-to-all synapses, so each cycle delivers N * N events."""
    n = 300
    params = lif_params(n, 60e-9, refract=0.0)  # v_tmp ~ 15 mV per cycle: reset to threshold in one step
    params[:, 0] = -0.049
    k = np.arange(n * n)
    src, dst = k // n, k % n
    w = np.where(k % 5 == 0, -1e-11, 2e-11)
    r = check(params, src, dst, w, np.full(n * n, 2), 60)
    assert r["fire_count"].min() == 60


def test_silent_sources_and_unreached_targets():
    """Half the neurons have no out-synapses, a quarter none in."""
    n = 800
    rng = np.random.default_rng(5)
    params = lif_params(n, rng.uniform(0.0, 0.4e-9, n), seed=5)
    s = 6000
    src = rng.integers(0, n // 2, s)
    dst = rng.integers(n // 4, n, s)
    w = rng.uniform(-3e-10, 4e-10, s)
    d = rng.integers(1, 9, s)
    r = check(params, src, dst, w, d, 500)
    assert r["fire_count"][: n // 4].sum() > 0


def test_raster_into_caller_buffer():
    """raster(out=...) reads into the caller's buffer (views into it) and gives the same
    spikes as a fresh read; a buffer too small is not used."""
    n = 500
    rng = np.random.default_rng(3)
    params = lif_params(n, rng.uniform(0.1e-9, 0.4e-9, n), seed=3)
    s = 3000
    eng = B.Engine.from_arrays(params, rng.integers(0, n, s).astype(np.int32), rng.integers(0, n, s).astype(np.int32),
                               rng.uniform(-2e-10, 3e-10, s).astype(np.float32), rng.integers(1, 7, s).astype(np.int32),
                               DT)
    eng.record(300, n * 300)
    eng.run(300)
    fresh = eng.raster()
    total = sum(len(r) for r in fresh)
    assert total > 0
    buf = np.full(total + 10, -7, np.int32)
    into = eng.raster(out=buf)
    assert all(np.array_equal(x, y) for x, y in zip(fresh, into)) and len(into) == len(fresh)
    assert np.shares_memory(into[-1], buf) or len(into[-1]) == 0
    assert np.array_equal(buf[:total], np.concatenate(fresh)) and buf[total] == -7
    small = np.zeros(max(total - 1, 1), np.int32)
    again = eng.raster(out=small)
    assert all(np.array_equal(x, y) for x, y in zip(fresh, again)) and not small.any()
    eng.close()


def test_bounded_wait_times_out_with_a_device_error():
    """Failure detection without a GPU fault: a tile whose finisher count is preset
    (bsim_stall_tile) makes every block that finishes a piece of it wait for a
    store that never comes. The wait gives up after its bound, the step raises
    BSIM_DEVERR_TIMEOUT and ends, bsim_run returns BSIM_ERR_DEVICE naming the code,
    later steps do not run (state unchanged), and the buffers stay readable."""
    from bsim_b200 import workloads as W
    import time
    sp = W.cuba(4, 500, 500, 6, seed=9)
    eng = B.Engine.generated(sp, DT, opts=B.options(delivery=B.DELIVERY_TILE))
    eng.run(30)
    before = eng.state()["v"].copy()
    with pytest.raises(B.BsimError):
        B._check(B.lib().bsim_stall_tile(eng._h, eng.info().n_neurons))  # no such tile
    B._check(B.lib().bsim_stall_tile(eng._h, 0))
    t0 = time.perf_counter()
    with pytest.raises(B.BsimError) as err:
        eng.run(1)
    assert "bounded wait" in str(err.value) and time.perf_counter() - t0 < 30.0
    after_fault = eng.state()["v"].copy()
    assert not np.array_equal(after_fault, before)  # the stalled step itself ran to its end
    with pytest.raises(B.BsimError):
        eng.run(5)
    assert np.array_equal(eng.state()["v"], after_fault)  # nothing ran after the flag
    assert eng.fire_count().shape == (sp.n_pop * sp.pop_size,)
    eng.close()


@pytest.mark.parametrize("tile_size", [1024, 256])
def test_tiled_segment_lengths_around_the_bank_ordering_limit(tile_size):
    """The tiled copy reorders the entries of each (tile, source, delay) segment of up
    to 256 entries by shared-memory bank and keeps longer ones in target order. Sources
    with 1, 2, 3, 255, 256, 257 and 300 targets at one delay (padded to even lengths,
    excitatory and inhibitory mixed, so both counter halves' banks occur), in one tile
    and in tiles of 256 targets: spikes, state and events equal the oracle's."""
    n = 700
    rng = np.random.default_rng(11)
    params = lif_params(n, rng.uniform(0.15e-9, 0.35e-9, n), seed=11)
    params[:7, 9] = 3e-9  # the long-row sources are driven to fire regularly
    src, dst, w, d = [], [], [], []
    for s_id, k in enumerate([1, 2, 3, 255, 256, 257, 300]):
        tg = np.sort(rng.choice(n, k, replace=False))
        src += [s_id] * k
        dst += tg.tolist()
        w += rng.uniform(-6e-11, 9e-11, k).tolist()
        d += [1 + s_id % 3] * k
    m = 3000  # background synapses so that the sources fire
    src += rng.integers(0, n, m).tolist()
    dst += rng.integers(0, n, m).tolist()
    w += rng.uniform(-2e-10, 3e-10, m).tolist()
    d += rng.integers(1, 5, m).tolist()
    src, dst = np.asarray(src, np.int32), np.asarray(dst, np.int32)
    w, d = np.asarray(w, np.float32), np.asarray(d, np.int32)
    steps = 400
    eng = B.Engine.from_arrays(params, src, dst, w, d, DT,
                               opts=B.options(delivery=B.DELIVERY_TILE, tile_size=tile_size))
    eng.record(steps, n * steps)
    eng.run(steps)
    ras = eng.raster()
    ref = oracle.run(params, src, dst, w, d, DT, steps, record_steps=steps, acc_mode=oracle.ACC_FIXED,
                     qexp=int(eng.qexp()[0]), raster_cap=n * steps)
    assert sum(len(r) for r in ras) > 0
    for t in range(steps):
        assert np.array_equal(ras[t], ref["raster"][t]), t
    assert np.array_equal(eng.fire_count(), ref["fire_count"])
    assert np.array_equal(eng.state()["v"], ref["final_state"][:, 0])
    assert eng.info().events_total == ref["events_per_step"].sum()
    assert (ref["fire_count"][:7] >= 10).all()  # every long-row source spikes repeatedly
    eng.close()
