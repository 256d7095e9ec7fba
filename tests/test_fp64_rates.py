"""Population rates of the engine against the double-precision reference, per
configuration: the BASELINE workloads' generator networks (the 10 x 1,000 one at
full size, the 1e6- and 2e6-neuron ones as scaled replicas with the same
populations, rates and delays) run by the engine (fp32 state, exact fixed-point
input sums) and by the oracle's double build in reference order (the
reference's -DUSE_DOUBLE STSim semantics, src/neuron/lif/LIFENeuron.cpp:114-160).

The double run takes the networks' random draws (v_init, i_offset, weights) as
generated and the preset constants as the decimal values a program passes to
the double build (so tau_refrac / dt truncates to the same step count as in the
float build: 2e-4 s / 1e-4 s is 2 steps in double, and 1.99999995 in double from
the float-rounded value).

Run as a script (no GPU) it prints the same measures for the oracle's
fixed-point float mode, which the GPU parity tests show to be bit-identical to
the engine, and for the reference's float build."""
import math
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from bsim_b200 import workloads as W  # noqa: E402
from oracle import oracle  # noqa: E402

DT = 1e-4
# name -> (spec factory, tau_refrac as written, cycles compared)
CONFIGS = {
    "c0_10x1000_100Hz_d6": (lambda: W.cuba(10, 1000, 100, 6, seed=1), 2e-3, 2000),
    "c1_replica_100x200_d6": (lambda: W.scaled(W.plain_1m(1)[0][0], 200), 0.5e-3, 1000),
    "c2_replica_50x400_2kHz_d50": (lambda: W.scaled(W.dense_1m(1)[0][0], 400), 0.2e-3, 500),
    "c4_replica_200x100_square_d20": (lambda: W.scaled(W.predicted_2m(1)[0][0], 100), 0.5e-3, 1000),
}
TOTAL_TOL = 0.01  # whole-network rate, relative
POP_TOL = 0.05    # each population, relative to max(its double-precision rate, 10 Hz)


def f64_params(params, tau_refrac):
    """Per-neuron draws as generated; the preset constants as exact decimals."""
    p = params.astype(np.float64)
    p[:, 1] = -65e-3  # v_rest
    p[:, 2] = -65e-3  # v_reset
    p[:, 3] = 0.25e-9  # cm
    p[:, 4] = 20e-3  # tau_m
    p[:, 5] = tau_refrac
    p[:, 6] = 5e-3  # tau_syn_E
    p[:, 7] = 10e-3  # tau_syn_I
    p[:, 8] = -50e-3  # v_thresh
    return p


def drive(spec, g):
    """The square-wave drive's second parameter set (i_offset x drive_scale), or None."""
    if spec.drive_half_period <= 0:
        return None
    hi = g["params"].copy()
    hi[:, 9] = (g["params"][:, 9] * np.float32(spec.drive_scale)).astype(np.float32)
    return hi


def run_f64(spec, g, tau_refrac, steps):
    hi = drive(spec, g)
    kw = {} if hi is None else dict(params_alt=f64_params(hi, tau_refrac), half_period=int(spec.drive_half_period))
    return oracle.run(f64_params(g["params"], tau_refrac), g["src"], g["dst"], g["weight"], g["delay_steps"], DT,
                      steps, acc_mode=oracle.ACC_SEQUENTIAL, dtype=np.float64, **kw)["fire_count"]


def run_f32(spec, g, steps, mode, qexp=None):
    hi = drive(spec, g)
    kw = {} if hi is None else dict(params_alt=hi, half_period=int(spec.drive_half_period))
    return oracle.run(g["params"], g["src"], g["dst"], g["weight"], g["delay_steps"], np.float32(DT), steps,
                      acc_mode=mode, qexp=qexp, **kw)["fire_count"]


def pop_rates(fire_count, spec, steps):
    return fire_count.reshape(spec.n_pop, -1).sum(1).astype(np.float64) / (spec.pop_size * steps * DT)


def rate_errors(r, r64):
    """(whole-network relative error, largest and median per-population error)."""
    total = abs(r.sum() - r64.sum()) / r64.sum()
    per = np.abs(r - r64) / np.maximum(r64, 10.0)
    return total, float(per.max()), float(np.median(per))


def host_qexp(g):
    """The engine's fixed-point exponent for one network (largest in-degree, largest |w|)."""
    m = int(np.bincount(g["dst"], minlength=g["params"].shape[0]).max())
    e_w = math.frexp(float(np.abs(g["weight"]).max()))[1]
    return 61 - max(0, math.ceil(math.log2(m))) - e_w


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CONFIGS))
def test_engine_rates_vs_double_reference(name):
    import bsim_b200 as B
    make, tref, steps = CONFIGS[name]
    spec = make()
    g = B.gen_host(spec)
    eng = B.Engine.generated(spec, np.float32(DT))
    eng.run(steps)
    r = pop_rates(eng.fire_count(), spec, steps)
    r64 = pop_rates(run_f64(spec, g, tref, steps), spec, steps)
    total, worst, median = rate_errors(r, r64)
    print("%s: whole network %.4f, worst population %.4f, median %.4f" % (name, total, worst, median))
    assert total <= TOTAL_TOL and worst <= POP_TOL


def test_double_constants_keep_refractory_steps():
    """The decimal constants give the double build the refractory step counts of
    the float build (the truncation (int)(tau_refrac / dt) of each preset)."""
    for _, tref, _ in CONFIGS.values():
        f32 = int(np.float32(tref) / np.float32(DT))
        f64 = int(tref / DT)
        assert f32 == f64


if __name__ == "__main__":
    oracle.build()
    print("config | cycles | mean rate (double) | engine = fixed-point float: whole / worst pop / median pop"
          " | reference float build: whole / worst pop / median pop")
    for name, (make, tref, steps) in CONFIGS.items():
        spec = make()
        g = oracle.gen_host(spec)
        r64 = pop_rates(run_f64(spec, g, tref, steps), spec, steps)
        rf = pop_rates(run_f32(spec, g, steps, oracle.ACC_FIXED, qexp=host_qexp(g)), spec, steps)
        rs = pop_rates(run_f32(spec, g, steps, oracle.ACC_SEQUENTIAL), spec, steps)
        print("%s | %d | %.1f Hz | %.4f / %.4f / %.4f | %.4f / %.4f / %.4f"
              % ((name, steps, r64.mean()) + rate_errors(rf, r64) + rate_errors(rs, r64)))
