"""The firing predictor: its MLP kernels against a float64 CPU reference, its
use inside the step (scheduling only: rasters unchanged), and what the trained
network gains over the schedule without it (persistence of the last count)."""
import numpy as np
import pytest

import bsim_b200 as B
from bsim_b200 import predictor as PR
from bsim_b200 import workloads as W
from oracle import mlp_oracle

DT = np.float32(1e-4)


def test_cpu_mlp_gradient_matches_finite_differences():
    """Pins the numpy reference itself (float64 central differences)."""
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.3, B.MLP_PARAMS)
    x = rng.normal(0, 1, (16, 9))
    y = rng.normal(0, 1, 16)
    _, g = mlp_oracle.loss_and_grad(p, x, y)
    for i in rng.choice(B.MLP_PARAMS, 40, replace=False):
        e = np.zeros_like(p)
        e[i] = 1e-6
        num = (mlp_oracle.loss_and_grad(p + e, x, y)[0] - mlp_oracle.loss_and_grad(p - e, x, y)[0]) / 2e-6
        assert abs(num - g[i]) <= 1e-6 + 1e-5 * abs(num)


def test_mlp_init_is_deterministic():
    a, b = B.mlp_init(5), B.mlp_init(5)
    assert np.array_equal(a, b) and not np.array_equal(a, B.mlp_init(6))
    assert np.all(a[576:640] == 0)  # b1


def test_fit_costs_linear_model_and_its_guards():
    """The delivery cost model (ns per cycle = a + b x events) fitted from per-chunk
    measurements: exact on linear data; a negative slope falls back to the mean cost,
    a negative intercept to a fit through the origin (both coefficients stay >= 0)."""
    e = np.array([1e6, 3e6, 7e6, 2e7])
    assert np.allclose(PR.fit_costs(e, 5e4 + 4e-3 * e), [5e4, 4e-3])
    a, b = PR.fit_costs(e, 9e4 - 1e-3 * e)
    assert b == 0.0 and a == pytest.approx((9e4 - 1e-3 * e).mean())
    t = -2e4 + 6e-3 * e
    a, b = PR.fit_costs(e, t)
    assert a == 0.0 and b == pytest.approx((e * t).sum() / (e * e).sum())


@pytest.mark.gpu
def test_mlp_kernels_match_cpu_reference():
    rng = np.random.default_rng(1)
    p = B.mlp_init(3)
    x = rng.uniform(0, 2, (2048, 9)).astype(np.float32)
    y = rng.uniform(0, 2, 2048).astype(np.float32)
    yf = B.mlp_forward(p, x)
    assert np.allclose(yf, mlp_oracle.forward(p, x), rtol=1e-5, atol=1e-6)
    g, loss = B.mlp_grad(p, x, y)
    l_ref, g_ref = mlp_oracle.loss_and_grad(p, x, y)
    assert abs(loss - l_ref) <= 1e-5 * abs(l_ref)
    assert np.linalg.norm(g - g_ref) <= 1e-4 * np.linalg.norm(g_ref)


@pytest.mark.gpu
def test_mlp_training_reduces_loss():
    rng = np.random.default_rng(2)
    x = rng.uniform(0, 1, (8192, 9)).astype(np.float32)
    y = (x[:, :8].mean(1) * 1.5 + 0.1).astype(np.float32)
    p0 = B.mlp_init(1)
    _, l0 = B.mlp_grad(p0, x, y)
    p1, l1 = B.mlp_train(p0, x, y, epochs=20, batch=256, lr=2e-3)
    assert l1 < 0.05 * l0


def driven(seed):
    sp = W.cuba(10, 1000, 500, 6, seed=seed, i_max=2e-9)
    sp.drive_scale = 8.0
    sp.drive_half_period = 500
    return sp


@pytest.fixture(scope="module")
def trained():
    counts, size, indeg = PR.collect([driven(1)], 6000, DT)
    x, y = PR.features(counts, size, indeg)
    params, loss = PR.train(x, y, epochs=15, batch=512, lr=2e-3)
    return params, loss


@pytest.mark.gpu
def test_trained_predictor_beats_persistence(trained):
    """On a different seed of the square-wave driven network, the MLP's error on
    next-but-one-cycle population rates is below that of persistence (the last
    count) and of the 8-cycle mean, the schedules without a learned model."""
    params, _ = trained
    counts, size, indeg = PR.collect([driven(2)], 4000, DT)
    x, y = PR.features(counts, size, indeg)
    mae_mlp = np.abs(B.mlp_forward(params, x).clip(0) - y).mean()
    mae_last = np.abs(x[:, 0] - y).mean()
    mae_mean = np.abs(x[:, :8].mean(1) - y).mean()
    assert mae_mlp < mae_last and mae_mlp < mae_mean


@pytest.mark.gpu
def test_predictor_scheduling_keeps_rasters_identical(trained):
    params, _ = trained
    sp = driven(3)
    plain = B.Engine.generated(sp, DT)
    auto = B.Engine.generated(sp, DT, opts=B.options(delivery=B.DELIVERY_AUTO))
    auto.enable_pop_stats(64)
    # a cost model under which the cheaper mode changes with the load
    auto.set_predictor(params, tolerance=0.3, cost_push=[0.0, 1.0], cost_tile=[20000.0, 0.5])
    n = sp.n_pop * sp.pop_size
    for e in (plain, auto):
        e.record(1200, n * 1200)
        e.run(1200)
    ra, rb = plain.raster(), auto.raster()
    assert all(np.array_equal(a, b) for a, b in zip(ra, rb))
    assert np.array_equal(plain.state()["v"], auto.state()["v"])
    st = auto.predictor_stats()
    assert st.cycles == 1200
    assert 0 < st.tile_cycles < st.cycles  # the choice switched with the square wave
    assert st.fallbacks < 0.5 * st.cycles
    assert st.abs_err_sum < 0.5 * st.actual_sum


@pytest.mark.gpu
def test_autotune_keeps_dynamics(trained):
    sp = W.cuba(10, 1000, 100, 6, seed=4)
    a = B.Engine.generated(sp, DT, opts=B.options(build_tiles=1))
    b = B.Engine.generated(sp, DT)
    r = a.autotune(20)
    assert r.candidates >= 4 and r.delivery in (B.DELIVERY_PUSH, B.DELIVERY_TILE)
    steps = a.info().steps_done
    b.run(steps)
    a.run(300)
    b.run(300)
    assert np.array_equal(a.state()["v"], b.state()["v"])


@pytest.mark.gpu
@pytest.mark.parametrize("opts", [dict(delivery=B.DELIVERY_AUTO), dict(delivery=B.DELIVERY_TILE),
                                  dict(), dict(delivery=B.DELIVERY_PULL)])
def test_population_degrees_from_every_synapse_copy(opts):
    """Mean in/out-degree per population as the engine derives them (from the
    pull rows, the push rows or the tiled copy, whichever it holds) against the
    host generator's synapse list, for two networks packed in one engine."""
    specs = [W.cuba(4, 300, 100, 6, seed=61), W.cuba(3, 400, 500, 12, seed=62)]
    eng = B.Engine.generated(specs, DT, opts=B.options(**opts))
    size, indeg, outdeg = eng.pop_info()
    want_in, want_out, want_size = [], [], []
    for sp in specs:
        g = B.gen_host(sp)
        pops = g["pop"]
        P = sp.n_pop
        want_size += [sp.pop_size] * P
        want_in += list(np.bincount(pops[g["dst"]], minlength=P) / sp.pop_size)
        want_out += list(np.bincount(pops[g["src"]], minlength=P) / sp.pop_size)
    assert list(size) == want_size
    assert np.allclose(indeg, want_in, rtol=1e-6) and np.allclose(outdeg, want_out, rtol=1e-6)


@pytest.mark.gpu
def test_autotune_of_a_tiled_engine_keeps_dynamics():
    """A tiled-only engine never clears its accumulator planes; the autotuner's trials
    switch it to clearing (push adds into the planes) in mid-run. The spikes and state
    afterwards equal a push engine's over the same cycles."""
    sp = W.cuba(10, 1000, 500, 6, seed=8)
    a = B.Engine.generated(sp, DT, opts=B.options(delivery=B.DELIVERY_TILE))
    b = B.Engine.generated(sp, DT)
    a.run(150)
    r = a.autotune(5)
    assert r.candidates >= 4
    steps = a.info().steps_done
    b.run(steps)
    a.run(300)
    b.run(300)
    assert np.array_equal(a.state()["v"], b.state()["v"])
    assert np.array_equal(a.fire_count(), b.fire_count())


@pytest.mark.gpu
def test_auto_without_tiled_copy_pushes_every_cycle(trained):
    params, _ = trained
    sp = driven(5)
    plain = B.Engine.generated(sp, DT)
    auto = B.Engine.generated(sp, DT, opts=B.options(delivery=B.DELIVERY_AUTO, build_tiles=-1))
    auto.enable_pop_stats(64)
    auto.set_predictor(params, tolerance=0.3, cost_push=[1e6, 1.0], cost_tile=[0.0, 0.0])
    for e in (plain, auto):
        e.run(600)
    assert np.array_equal(plain.state()["v"], auto.state()["v"])
    assert auto.predictor_stats().tile_cycles == 0
    with pytest.raises(B.BsimError):
        B.Engine.generated(sp, DT, opts=B.options(delivery=B.DELIVERY_TILE, build_tiles=-1))


@pytest.mark.gpu
def test_exact_schedule_switches_modes_and_keeps_dynamics():
    """AUTO delivery under the exact schedule (no predictor: the cost models on the
    delivered window's exact spike count) on a square-wave-driven network: both
    modes are used and the spikes equal the plain push run's."""
    import bsim_b200 as B
    from bsim_b200 import workloads as W
    sp = W.cuba(8, 600, 500, 20, seed=71, i_max=2.5e-9)
    sp.drive_scale, sp.drive_half_period = 32.0, 100
    dt = np.float32(1e-4)
    plain = B.Engine.generated(sp, dt)
    plain.record(600, 600 * 4800)
    plain.run(600)
    spikes = np.array([len(r) for r in plain.raster()], np.float64)
    # the exact schedule's work: the mean spikes of the delivered window (20 cycles)
    # times the mean out-degree; put the crossover at the median window
    win = np.array([spikes[max(0, t - 20):t].sum() / 20.0 for t in range(600)])
    auto = B.Engine.generated(sp, dt, opts=B.options(delivery=B.DELIVERY_AUTO))
    inf = auto.info()
    work = float(np.median(win[20:])) * inf.n_synapses / inf.n_neurons
    auto.set_predictor(None, cost_push=[0.0, 1.0], cost_tile=[work, 0.0])
    auto.run(600)
    st = auto.predictor_stats()
    assert st.cycles == 600 and st.fallbacks == 0
    assert 60 < st.tile_cycles < 540
    assert np.array_equal(auto.fire_count(), plain.fire_count())
    assert np.array_equal(auto.state()["v"], plain.state()["v"])
