"""CPU-side checks of the engine library: it loads, exports every symbol the
public header declares, and its host-side logic (generator, synapse reset,
argument validation) behaves; no GPU compute is called here."""
import ctypes
import os
import re

import numpy as np
import pytest

import bsim_b200 as B
from bsim_b200 import workloads as W
from oracle import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    syms = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            syms |= set(re.findall(r"^\s*(?:int|const char \*|void)\s*\*?\s*(bsim_\w+)\s*\(", txt, re.M))
    return syms


def test_library_exports_every_declared_symbol():
    L = B.lib()
    syms = header_symbols()
    assert {"bsim_create", "bsim_run", "bsim_destroy"} <= syms
    for s in syms:
        assert hasattr(L, s), s
    assert set(B.EXPORTS) <= syms


def test_options_default():
    o = B.options()
    assert o.accumulate == B.ACC_EXACT and o.delivery == B.DELIVERY_PUSH and o.graph_steps == 64


def test_generator_is_deterministic_and_in_creation_order():
    spec = W.cuba(6, 200, 100, 6, seed=11)
    a = B.gen_host(spec)
    b = B.gen_host(spec)
    for k in a:
        assert np.array_equal(a[k], b[k])
    n = 6 * 200
    src, dst, w, d = a["src"], a["dst"], a["weight"], a["delay_steps"]
    assert src.min() >= 0 and src.max() < n and dst.min() >= 0 and dst.max() < n
    assert d.min() >= 1 and d.max() <= 6
    # creation order: projections, then source-major / target-minor inside each
    sp, tp = src // 200, dst // 200
    proj_start = np.flatnonzero(np.r_[True, (sp[1:] != sp[:-1]) | (tp[1:] != tp[:-1])])
    for s0, s1 in zip(proj_start, np.r_[proj_start[1:], len(src)]):
        key = src[s0:s1].astype(np.int64) * n + dst[s0:s1]
        assert np.all(np.diff(key) > 0)
    # chain projections first (k -> k+1, k = 0..P-2), then remote ones
    pairs = [(int(sp[i]), int(tp[i])) for i in proj_start]
    assert pairs[:5] == [(k, k + 1) for k in range(5)]
    assert len(pairs) == 5 + round(0.2 * 6)
    # sizes and statistics: p = 0.1, 80 % excitatory, |w_inh| up to 4 w_max
    assert abs(len(src) / (len(pairs) * 200 * 200) - 0.1) < 0.01
    assert abs((w >= 0).mean() - 0.8) < 0.02
    assert w.max() < 1e-10 and w.min() >= -4e-10
    p = a["params"]
    assert np.all((p[:, 9] >= 0) & (p[:, 9] < 3.2e-9))
    assert np.all((p[:, 0] >= -65e-3) & (p[:, 0] < -50e-3))


def test_synapse_reset_matches_oracle():
    rng = np.random.default_rng(3)
    delay = (rng.integers(1, 7, 500) * np.float32(1e-4) + rng.choice([0, 0.4e-4], 500)).astype(np.float32)
    w = rng.normal(0, 1e-10, 500).astype(np.float32)
    tau = rng.choice([5e-3, 10e-3], 500).astype(np.float32)
    st, wo = B.synapse_reset(delay, w, tau, np.float32(1e-4))
    st_o, wo_o = oracle.syn_reset(delay, w, tau, np.float32(1e-4))
    assert np.array_equal(st, st_o) and np.array_equal(wo, wo_o)


def test_create_rejects_bad_input_before_touching_a_gpu():
    params = np.zeros((4, 10), np.float32)
    with pytest.raises(B.BsimError) as ei:
        B.Engine.from_arrays(params, [0], [1], [1e-10], [0], 1e-4)
    assert ei.value.code == -4  # BSIM_ERR_DELAY
    with pytest.raises(B.BsimError) as ei:
        B.Engine.from_arrays(params, [0], [7], [1e-10], [1], 1e-4)
    assert ei.value.code == -1
    with pytest.raises(B.BsimError) as ei:
        B.Engine.from_arrays(params, [0], [1], [1e-10], [1], 1e-4, instance=[0, 1, 0, 0])
    assert ei.value.code == -1
    with pytest.raises(B.BsimError):
        B.Engine.generated(W.cuba(2, 10, 100, 65), 1e-4)  # device builder: delays up to 64
