"""The C++ front end (include/BSim.h): a program written against the reference's
user API compiles against it and, on a GPU, reproduces the reference's outputs
(GFire.count, and with -DLOG_DATA the GSim.log raster and g_v.data traces)."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import bsim_b200 as B
import netio
from oracle import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "lif_api_demo.cpp")
GOLDEN = np.load(os.path.join(ROOT, "tests", "golden", "lif_unit_v.npz"))


def compile_demo(out, log_data, src=SRC):
    cmd = ["g++", "-std=c++11", "-O2", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "include"), src,
           "-L" + os.path.dirname(B.LIB_PATH), "-lbsim_b200", "-Wl,-rpath," + os.path.dirname(B.LIB_PATH), "-o", out]
    if log_data:
        cmd.insert(1, "-DLOG_DATA")
    subprocess.run(cmd, check=True)


@pytest.fixture(scope="module")
def demos(tmp_path_factory):
    d = tmp_path_factory.mktemp("cppdemo")
    plain, logged = str(d / "demo"), str(d / "demo_log")
    compile_demo(plain, False)
    compile_demo(logged, True)
    return plain, logged


def test_reference_style_program_compiles(demos):
    assert all(os.path.exists(p) for p in demos)


def oracle_unit(which):
    net = netio.lif_unit_net(which)
    st, w = oracle.syn_reset(net["delay"], net["weight"], netio.syn_tau(net), np.float32(1e-4))
    return oracle.run(net["params"], net["src"], net["dst"], w, st, np.float32(1e-4), 1000, record_steps=1000,
                      rec_ids=np.arange(30))


@pytest.mark.gpu
@pytest.mark.parametrize("which", [1, 2, 3, 4])
@pytest.mark.parametrize("acc", ["exact", "ordered", "exact-tile"])
def test_sgsim_outputs_match_reference(demos, which, acc):
    ref = oracle_unit(which)
    env = dict(os.environ, BSIM_ACCUMULATE=acc.split("-")[0])
    if acc.endswith("tile"):
        env["BSIM_DELIVERY"] = "tile"
    with tempfile.TemporaryDirectory() as d:
        subprocess.run([demos[1], str(which)], cwd=d, check=True, env=env, stdout=subprocess.DEVNULL)
        count = np.loadtxt(os.path.join(d, "GFire.count"), dtype=np.int64)
        v = np.loadtxt(os.path.join(d, "g_v.data"))
        ie = np.loadtxt(os.path.join(d, "g_ie.data"))
        ii = np.loadtxt(os.path.join(d, "g_ii.data"))
        ine = np.loadtxt(os.path.join(d, "g_input_e.data"))
        ini = np.loadtxt(os.path.join(d, "g_input_i.data"))
        raster = [np.array(line.split(), dtype=np.int32) for line in open(os.path.join(d, "GSim.log"))]
        info = open(os.path.join(d, "GSim.info")).read()
    assert "NeuronNum: 30, SynapseNum: 200" in info
    # the per-cycle files come from the on-device trace: one line per cycle, one value per neuron
    for arr in (v, ie, ii, ine, ini):
        assert arr.shape == (1000, 30)
    printed = lambda x: np.array([float("%.10f" % y) for y in np.ravel(x)])
    # synaptic currents after the last cycle: printed digit for digit in reference order; with
    # exact sums they drift from the sequential ones by the rounding of 1,000 cycles of
    # accumulation with tau_syn = 1 s (relative 1e-4), while v stays within 3.5e-7 V (below)
    tol = 1.01e-10 if acc == "ordered" else 1.01e-10 + 1e-4 * np.abs(printed(ref["final_state"][:, 1:3]))
    fin = np.stack([ie[-1], ii[-1]], 1).ravel()
    assert np.all(np.abs(fin - printed(ref["final_state"][:, 1:3])) <= tol)
    assert ine.min() >= 0 and ini.max() <= 0
    assert np.array_equal(count, ref["fire_count"])
    assert len(raster) == 1000 and all(np.array_equal(a, b) for a, b in zip(raster, ref["raster"]))
    assert np.abs(v - GOLDEN["unit%d" % which]).max() < 3.5e-7
    if acc == "ordered":
        printed = np.array([float("%.10f" % x) for x in ref["v_trace"].ravel()]).reshape(v.shape)
        assert np.array_equal(v, printed)


@pytest.mark.gpu
def test_sgsim_plain_build_writes_fire_count(demos):
    ref = oracle_unit(2)
    with tempfile.TemporaryDirectory() as d:
        subprocess.run([demos[0], "2"], cwd=d, check=True, stdout=subprocess.DEVNULL)
        count = np.loadtxt(os.path.join(d, "GFire.count"), dtype=np.int64)
    assert np.array_equal(count, ref["fire_count"])


DRIVE_SRC = os.path.join(ROOT, "tests", "cpp", "drive_api_demo.cpp")


@pytest.fixture(scope="module")
def drive_demo(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("cppdrive") / "drive_demo")
    compile_demo(out, False, DRIVE_SRC)
    return out


def test_drive_program_compiles(drive_demo):
    assert os.path.exists(drive_demo)


def drive_demo_oracle(seed):
    """The network of tests/cpp/drive_api_demo.cpp in flat form, run by the oracle."""
    NC, NP, NL = 4, 6, 8
    params = np.zeros((NC + NP + NL, 10), np.float32)
    params[:NC, :3] = [0.02, 0.0, 0.15]
    params[NC:NC + NP, :4] = [40.0, 1e-3, 0.005, 1000.0]
    params[NC + NP:] = [-0.065, -0.065, -0.065, 0.25e-9, 20e-3, 2e-3, 5e-3, 10e-3, -0.050, 0.1e-9]
    kind = np.array([1] * NC + [2] * NP + [0] * NL, np.uint8)
    i_c, i_p = np.arange(NC * NL), np.arange(NP * NL)
    src = np.concatenate([i_c // NL, NC + i_p // NL]).astype(np.int32)
    dst = np.concatenate([NC + NP + i_c % NL, NC + NP + i_p % NL]).astype(np.int32)
    wc = np.float32(1e-9) + np.float32(1e-10) * (i_c % 7).astype(np.float32)
    wp = np.float32(2e-9) - np.float32(1e-10) * (i_p % 5).astype(np.float32)
    delay = np.concatenate([np.full(NC * NL, 2e-4), np.full(NP * NL, 5e-4)]).astype(np.float32)
    tau = np.concatenate([np.full(NC * NL, 1e-3), np.full(NP * NL, 1e-3)]).astype(np.float32)
    st, w = oracle.syn_reset(delay, np.concatenate([wc, wp]), tau, np.float32(1e-4))
    return oracle.run(params, src, dst, w, st, np.float32(1e-4), 2000, kind=kind, input_seed=seed)


@pytest.mark.gpu
def test_drive_program_fire_count_matches_oracle(drive_demo):
    """GFire.count of the program equals the oracle's spike counts (Poisson draws
    seeded by BSIM_INPUT_SEED); the LIF population is driven into firing."""
    with tempfile.TemporaryDirectory() as d:
        env = dict(os.environ, BSIM_INPUT_SEED="3")
        subprocess.run([drive_demo], cwd=d, check=True, env=env, stdout=subprocess.DEVNULL)
        count = np.loadtxt(os.path.join(d, "GFire.count"), dtype=np.int64)
        info = open(os.path.join(d, "GSim.info")).read()
    ref = drive_demo_oracle(3)
    assert "NeuronTypeNum: 3" in info
    assert np.array_equal(count, ref["fire_count"])
    assert ref["fire_count"][10:].sum() > 0


# ---------------------------------------------------------------------------
# The reference's own example programs, compiled unchanged against include/BSim.h
# by `make -C oracle refprogs` (part of the build where the reference's sources are
# present): test/gpu/lif_unit{1..4}_test.cpp and test/gpu/standard_test.cpp.
# ---------------------------------------------------------------------------
PROGS = os.path.join(ROOT, "oracle", "_ref", "progs")
needs_progs = pytest.mark.skipif(not os.path.exists(os.path.join(PROGS, "standard_test.log")),
                                 reason="the reference's programs were not built (no reference sources)")


@pytest.mark.gpu
@needs_progs
@pytest.mark.parametrize("which", [1, 2, 3, 4])
def test_reference_unit_programs_unchanged(which):
    """lif_unit{k}_test.cpp of the reference, built with -DLOG_DATA: its g_v.data
    matches the reference's golden trace test/lif_unit{k}_test_v.std, its raster and
    GFire.count the oracle's."""
    ref = oracle_unit(which)
    with tempfile.TemporaryDirectory() as d:
        subprocess.run([os.path.join(PROGS, "lif_unit%d_test.log" % which)], cwd=d, check=True,
                       stdout=subprocess.DEVNULL)
        v = np.loadtxt(os.path.join(d, "g_v.data"))
        raster = [np.array(line.split(), dtype=np.int32) for line in open(os.path.join(d, "GSim.log"))]
        info = open(os.path.join(d, "GSim.info")).read()
    assert "NeuronNum: 30, SynapseNum: 200" in info
    assert v.shape == (1000, 30) and np.abs(v - GOLDEN["unit%d" % which]).max() < 3.5e-7
    assert len(raster) == 1000 and all(np.array_equal(a, b) for a, b in zip(raster, ref["raster"]))


@pytest.mark.gpu
@needs_progs
def test_reference_standard_test_program_unchanged():
    """standard_test.cpp of the reference (the all-to-all chain of its README's
    benchmark, 5 % preset) on a small depth: it builds, runs 1,000 cycles and writes
    the reference's output files; the network it builds has the size the program
    implies; ordered and exact accumulation (which differ only in rounding) give
    total spike counts within 5 % of each other."""
    depth, n = 8, 200
    counts = {}
    for acc in ("ordered", "exact"):
        with tempfile.TemporaryDirectory() as d:
            env = dict(os.environ, BSIM_ACCUMULATE=acc)
            subprocess.run([os.path.join(PROGS, "standard_test"), str(depth), str(n), "0.7", "0.9", "0.6", "0.2", "6"],
                           cwd=d, check=True, env=env, stdout=subprocess.DEVNULL)
            info = open(os.path.join(d, "GSim.info")).read()
            counts[acc] = np.loadtxt(os.path.join(d, "GFire.count"), dtype=np.int64)
    side = len(range(1, depth, 4))                  # inhibitory side populations
    conns = (depth - 1) + (depth // 6) + 2 * side  # chain, g1 -> g[i] for i % 6 == 0, side pairs
    assert "NeuronNum: %d, SynapseNum: %d" % ((depth + side) * n, conns * n * n) in info
    assert counts["exact"].shape == ((depth + side) * n,)
    assert counts["exact"].sum() > 0
    assert abs(int(counts["exact"].sum()) - int(counts["ordered"].sum())) <= 0.05 * counts["ordered"].sum()
