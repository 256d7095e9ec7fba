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


def compile_demo(out, log_data):
    cmd = ["g++", "-std=c++11", "-O2", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "include"), SRC,
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
@pytest.mark.parametrize("acc", ["exact", "ordered"])
def test_sgsim_outputs_match_reference(demos, which, acc):
    ref = oracle_unit(which)
    env = dict(os.environ, BSIM_ACCUMULATE=acc)
    with tempfile.TemporaryDirectory() as d:
        subprocess.run([demos[1], str(which)], cwd=d, check=True, env=env, stdout=subprocess.DEVNULL)
        count = np.loadtxt(os.path.join(d, "GFire.count"), dtype=np.int64)
        v = np.loadtxt(os.path.join(d, "g_v.data"))
        raster = [np.array(line.split(), dtype=np.int32) for line in open(os.path.join(d, "GSim.log"))]
        info = open(os.path.join(d, "GSim.info")).read()
    assert "NeuronNum: 30, SynapseNum: 200" in info
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
