"""On-device state trace (bsim_trace / bsim_read_trace), the engine's form of the
reference's LOG_DATA files g_v / g_ie / g_ii / g_input_e / g_input_i
(src/sim/SingleGPUSimulator.cu:150-206): the state after each cycle, recorded
inside the step, equals the state read back cycle by cycle, and the consumed
input equals the fixed-point oracle's sums."""
import numpy as np
import pytest

import bsim_b200 as B
from bsim_b200 import workloads as W

pytestmark = pytest.mark.gpu
DT = np.float32(1e-4)


@pytest.mark.parametrize("delivery", [B.DELIVERY_PUSH, B.DELIVERY_TILE])
def test_trace_equals_per_cycle_state(delivery):
    spec = W.cuba(6, 400, 500, 6, seed=61)
    a = B.Engine.generated(spec, DT, opts=B.options(delivery=delivery, graph_steps=16))
    b = B.Engine.generated(spec, DT, opts=B.options(delivery=delivery))
    a.run(37)
    b.run(37)
    first, count, steps = 150, 1700, 120
    a.trace(steps, first, count)
    a.run(steps)
    tr = a.read_trace()
    assert tr["v"].shape == (steps, count)
    for k in range(steps):
        b.run(1)
        s = b.state()
        assert np.array_equal(tr["v"][k], s["v"][first:first + count])
        assert np.array_equal(tr["i_E"][k], s["i_E"][first:first + count])
        assert np.array_equal(tr["i_I"][k], s["i_I"][first:first + count])
    # neurons that did not fire and were not refractory took the input: i_E(t) = CE * i_E(t-1) + in_E(t)
    assert np.abs(tr["in_E"]).max() > 0 and np.abs(tr["in_I"]).max() > 0
    assert tr["in_E"].min() >= 0 and tr["in_I"].max() <= 0


def test_trace_restart_and_partial_read():
    spec = W.cuba(3, 300, 100, 6, seed=62)
    e = B.Engine.generated(spec, DT)
    e.trace(50, 0, 900)
    e.run(20)
    assert e.read_trace()["v"].shape == (20, 900)
    e.run(40)
    assert e.read_trace()["v"].shape == (50, 900)
    e.trace(10, 100, 5)
    e.run(3)
    t = e.read_trace()
    assert t["v"].shape == (3, 5)
    assert np.array_equal(t["v"][-1], e.state()["v"][100:105])
