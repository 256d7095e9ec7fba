"""Pins the CPU oracle: against the reference's golden traces, its known-answer
constants, and (where the reference sources were built into oracle/_ref) the
reference's own single-thread simulator run on the same networks."""
import os
import tempfile

import numpy as np
import pytest

import netio
from oracle import oracle

GOLDEN = np.load(os.path.join(os.path.dirname(__file__), "golden", "lif_unit_v.npz"))


def run_unit(which, dtype):
    net = netio.lif_unit_net(which)
    st, w = oracle.syn_reset(net["delay"], net["weight"], netio.syn_tau(net), net["dt"], dtype=dtype)
    return oracle.run(net["params"], net["src"], net["dst"], w, st, net["dt"], net["steps"],
                      record_steps=net["steps"], rec_ids=np.arange(30), dtype=dtype)


@pytest.mark.parametrize("which", [1, 2, 3, 4])
def test_oracle_f64_reproduces_golden_exactly(which):
    """The double-precision restatement prints the reference's golden v traces
    (test/lif_unit{1..4}_test_v.std, "%.10lf") digit for digit."""
    r = run_unit(which, np.float64)
    printed = np.array([float("%.10f" % x) for x in r["v_trace"].ravel()]).reshape(r["v_trace"].shape)
    assert np.array_equal(printed, GOLDEN["unit%d" % which])


@pytest.mark.parametrize("which,spikes", [(1, 5000), (2, 6747), (3, 5000), (4, 3330)])
def test_oracle_f32_within_float_rounding_of_golden(which, spikes):
    """The float build stays within 3.5e-7 V of the golden traces with the same
    spike raster as the double build."""
    r32 = run_unit(which, np.float32)
    r64 = run_unit(which, np.float64)
    assert np.abs(r32["v_trace"].astype(np.float64) - GOLDEN["unit%d" % which]).max() < 3.5e-7
    assert sum(len(x) for x in r32["raster"]) == spikes
    for a, b in zip(r32["raster"], r64["raster"]):
        assert np.array_equal(a, b)


def test_lif_fold_known_answers():
    """Constant folding of LIFENeuron::reset for the lif_unit1 population-0
    neuron, against the known answers of the reference's test/lif_unit1_test.py:78-92."""
    net = netio.lif_unit_net(1)
    fold, rt = oracle.lif_reset(net["params"], np.float32(1e-4), dtype=np.float32)
    # fold columns: vm, CI, CE, C_I, C_E, v_tmp, i_I, i_E, v_thresh, v_reset, Cm
    np.testing.assert_array_almost_equal(fold[:, 10], [0.998001993] * 30)
    np.testing.assert_array_almost_equal(fold[:, 2], [0.999899983] * 30)
    np.testing.assert_array_almost_equal(fold[:, 1], [0.999899983] * 30)
    np.testing.assert_array_almost_equal(fold[:, 4], [0.000998942531] * 30)
    np.testing.assert_array_almost_equal(fold[:, 3], [0.000998942531] * 30)
    np.testing.assert_array_almost_equal(fold[:, 5], [0.00999003649] * 10 + [0.0] * 20)
    np.testing.assert_array_almost_equal(fold[:, 8], [0.0149999997] * 30)
    assert list(rt) == [0] * 30


def test_syn_reset_rescales_off_grid_delays():
    """StaticSynapse::reset: whole-step delays keep their weight; a delay of 1.5 dt
    rounds to 2 steps and scales the weight by expf(0.5 dt / tau)."""
    st, w = oracle.syn_reset([1e-4, 2e-4, 1.5e-4], [1.0, 1.0, 1.0], [1e-3, 1e-3, 1e-3], np.float32(1e-4))
    assert list(st) == [1, 2, 2]
    assert w[0] == 1.0 and w[1] == 1.0
    assert w[2] == np.float32(1.0) * np.exp(np.float32(0.5e-4) / np.float32(1e-3), dtype=np.float32)


def test_oracle_rejects_zero_delay():
    with pytest.raises(RuntimeError):
        oracle.run(np.zeros((2, 10)), [0], [1], [1.0], [0], 1e-4, 3)


def test_fixed_point_mode_matches_sequential_on_unit_nets():
    """With at most one input per target and step, the exact int64 sum equals the
    sequential sum bit for bit."""
    net = netio.lif_unit_net(2)
    st, w = oracle.syn_reset(net["delay"], net["weight"], netio.syn_tau(net), net["dt"])
    a = oracle.run(net["params"], net["src"], net["dst"], w, st, net["dt"], 1000, record_steps=1000,
                   rec_ids=np.arange(30))
    b = oracle.run(net["params"], net["src"], net["dst"], w, st, net["dt"], 1000, record_steps=1000,
                   rec_ids=np.arange(30), acc_mode=oracle.ACC_FIXED, qexp=40)
    assert all(np.array_equal(x, y) for x, y in zip(a["raster"], b["raster"]))
    assert np.abs(a["v_trace"] - b["v_trace"]).max() <= 1e-6


# ---------------------------------------------------------------------------
# Against the reference's own simulator (oracle/_ref, built from its sources)
# ---------------------------------------------------------------------------
needs_ref = pytest.mark.skipif(not (oracle.ref_available("f32") and oracle.ref_available("f64")),
                               reason="reference build oracle/_ref not present (make -C oracle ref)")


@needs_ref
@pytest.mark.parametrize("which", [1, 2, 3, 4])
@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_oracle_bit_exact_vs_reference_unit_nets(which, prec):
    net = netio.lif_unit_net(which)
    dtype = np.float32 if prec == "f32" else np.float64
    r = run_unit(which, dtype)
    with tempfile.TemporaryDirectory() as d:
        netio.write_net(os.path.join(d, "net.bin"), net, 1000, 1000, rec_ids=np.arange(30))
        ref = oracle.run_reference(os.path.join(d, "net.bin"), os.path.join(d, "out.bin"), prec, n=30, n_rec=30)
    assert np.array_equal(ref["v_trace"], r["v_trace"].astype(np.float64))
    for a, b in zip(ref["raster"], r["raster"]):
        assert np.array_equal(a, b)
    assert np.array_equal(ref["fire_count"], r["fire_count"])


def generated_net(spec):
    """A generated network in netio form: the float values the generator drew,
    delays as whole steps times dt (so StaticSynapse::reset keeps the weights)."""
    import bsim_b200 as B
    g = B.gen_host(spec)
    n = g["params"].shape[0]
    dt = np.float32(1e-4)
    return g, dict(params=g["params"].astype(np.float64), pop_size=np.full(spec.n_pop, spec.pop_size, np.int64),
                   pop_tau=np.tile([spec.tau_syn_E, spec.tau_syn_I], (spec.n_pop, 1)).astype(np.float64),
                   src=g["src"], dst=g["dst"], weight=g["weight"].astype(np.float64),
                   delay=(g["delay_steps"].astype(np.float32) * dt).astype(np.float64),
                   type=(g["weight"] < 0).astype(np.uint8), dt=float(dt), steps=0), n


@needs_ref
@pytest.mark.parametrize("shape", [(10, 300, 100, 6, 5), (8, 250, 2000, 50, 3), (6, 400, 500, 20, 11)])
def test_oracle_bit_exact_vs_reference_generated_net(shape):
    """Generated CUBA nets (10 x 300 at 100 Hz with delays U{1..6}; 8 x 250 at 2 kHz
    with delays U{1..50}; 6 x 400 at 500 Hz with delays U{1..20}): identical rasters,
    v and spike counts between the restatement and the reference simulator (float build)."""
    from bsim_b200 import workloads as W
    n_pop, size, rate, D, seed = shape
    spec = W.cuba(n_pop, size, rate, D, seed=seed)
    g, net, n = generated_net(spec)
    steps = 400
    rec = np.arange(0, n, 7, dtype=np.int32)
    with tempfile.TemporaryDirectory() as d:
        netio.write_net(os.path.join(d, "net.bin"), net, steps, steps, rec_ids=rec, dt=1e-4)
        ref = oracle.run_reference(os.path.join(d, "net.bin"), os.path.join(d, "out.bin"), "f32", n=n,
                                   n_rec=len(rec))
    st, w = oracle.syn_reset(net["delay"], net["weight"], netio.syn_tau(net), np.float32(1e-4))
    assert np.array_equal(st, g["delay_steps"]) and np.array_equal(w, g["weight"])
    r = oracle.run(g["params"], g["src"], g["dst"], g["weight"], g["delay_steps"], np.float32(1e-4), steps,
                   record_steps=steps, rec_ids=rec)
    assert sum(len(x) for x in r["raster"]) > 1000
    for a, b in zip(ref["raster"], r["raster"]):
        assert np.array_equal(a, b)
    assert np.array_equal(ref["v_trace"], r["v_trace"].astype(np.float64))
    assert np.array_equal(ref["fire_count"], r["fire_count"])


def test_oracle_generator_equals_engine_generator():
    """The oracle library's copy of the workload generator (used by the CPU
    baselines, which never load the engine) gives the engine's networks bit for bit."""
    import bsim_b200 as B
    from bsim_b200 import workloads as W
    for sp in (W.cuba(10, 300, 100, 6, seed=3), W.scaled(W.dense_1m(1)[0][0], 60),
               W.scaled(W.predicted_2m(1)[0][0], 40)):
        a, b = B.gen_host(sp), oracle.gen_host(sp)
        assert len(a["src"]) > 0
        for k in a:
            assert a[k].dtype == b[k].dtype and np.array_equal(a[k].view(np.uint32) if a[k].dtype == np.float32
                                                               else a[k], b[k].view(np.uint32)
                                                               if b[k].dtype == np.float32 else b[k])
