"""TEST INFRASTRUCTURE ONLY — Python handle on the CPU oracle (liboracle.so).

The oracle restates BSim's single-thread simulator for LIF_brian neurons and
static synapses (src/sim/SingleThreadSimulator.cpp:21-183 and the functions it
calls; see lif_oracle.h for the full list). Only tests/, __graft_entry__.smoke()
and bench.py's cpu_baseline leg may import this module, and only as the checker
or the timed CPU baseline, never as part of the product path.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

ACC_SEQUENTIAL = 0
ACC_FIXED = 1

_lib = None


def build():
    """Compile liboracle.so (and nothing else) with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)


def build_ref(ref_root):
    """Compile the reference's own simulator driver into oracle/_ref/ from the reference's
    source root `ref_root`, when its sources exist there."""
    if not os.path.isdir(os.path.join(ref_root, "src")):
        return False
    subprocess.run(["make", "-s", "-C", HERE, "ref", "REF=" + ref_root], check=True)
    return True


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        i64 = ctypes.c_int64
        for sfx, real in (("f32", ctypes.c_float), ("f64", ctypes.c_double)):
            f = getattr(L, "oracle_lif_reset_" + sfx)
            f.argtypes = [P, i64, real, P, P]
            f.restype = ctypes.c_int
            f = getattr(L, "oracle_syn_reset_" + sfx)
            f.argtypes = [P, P, P, i64, real, P, P]
            f.restype = ctypes.c_int
            f = getattr(L, "oracle_run_" + sfx)
            f.argtypes = [P, i64, P, P, P, P, i64, real, i64, ctypes.c_int, P, P]
            f.restype = ctypes.c_int
        L.oracle_poisson_draws.argtypes = [ctypes.c_uint64, ctypes.c_float, i64, P]
        L.oracle_poisson_draws.restype = ctypes.c_int
        L.oracle_gen_count.argtypes = [P, P, P]
        L.oracle_gen_count.restype = ctypes.c_int
        L.oracle_gen_host.argtypes = [P, P, P, P, P, P, P]
        L.oracle_gen_host.restype = ctypes.c_int
        _lib = L
    return _lib


class _Out(ctypes.Structure):
    _fields_ = [
        ("record_steps", ctypes.c_int64),
        ("fire_count", ctypes.c_void_p),
        ("raster_off", ctypes.c_void_p),
        ("raster_ids", ctypes.c_void_p),
        ("raster_cap", ctypes.c_int64),
        ("rec_ids", ctypes.c_void_p),
        ("n_rec", ctypes.c_int64),
        ("v_trace", ctypes.c_void_p),
        ("final_state", ctypes.c_void_p),
        ("spikes_per_step", ctypes.c_void_p),
        ("events_per_step", ctypes.c_void_p),
        ("params_alt", ctypes.c_void_p),
        ("half_period", ctypes.c_int64),
        ("kind", ctypes.c_void_p),
        ("instance", ctypes.c_void_p),
        ("input_seed", ctypes.c_uint64),
    ]


def _ptr(a):
    return None if a is None else a.ctypes.data


def lif_reset(params, dt, dtype=np.float32):
    """LIFENeuron::reset folding for every neuron: returns (fold[n,11], refrac_time[n])."""
    params = np.ascontiguousarray(params, dtype=dtype)
    n = params.shape[0]
    fold = np.zeros((n, 11), dtype=dtype)
    rt = np.zeros(n, dtype=np.int32)
    sfx = "f32" if dtype == np.float32 else "f64"
    rc = getattr(lib(), "oracle_lif_reset_" + sfx)(_ptr(params), n, dt, _ptr(fold), _ptr(rt))
    assert rc == 0
    return fold, rt


def syn_reset(delay_s, weight, tau_syn, dt, dtype=np.float32):
    """StaticSynapse::reset: (delay_steps int32[s], weight[s])."""
    d = np.ascontiguousarray(delay_s, dtype=dtype)
    w = np.ascontiguousarray(weight, dtype=dtype)
    t = np.ascontiguousarray(tau_syn, dtype=dtype)
    s = d.shape[0]
    st = np.zeros(s, dtype=np.int32)
    wo = np.zeros(s, dtype=dtype)
    sfx = "f32" if dtype == np.float32 else "f64"
    rc = getattr(lib(), "oracle_syn_reset_" + sfx)(_ptr(d), _ptr(w), _ptr(t), s, dt, _ptr(st), _ptr(wo))
    assert rc == 0
    return st, wo


def run(params, src, dst, weight, delay_steps, dt, steps, record_steps=0, rec_ids=None,
        acc_mode=ACC_SEQUENTIAL, qexp=None, dtype=np.float32, raster_cap=None, params_alt=None, half_period=0,
        kind=None, instance=None, input_seed=0):
    """Run the oracle. Returns a dict with fire_count, raster (list of arrays),
    v_trace [record_steps, n_rec], final_state [n, 4], spikes/events per step.
    params_alt / half_period: square-wave drive (params_alt's v_tmp in odd half periods).
    kind / instance / input_seed: input-drive neurons (0 LIF, 1 Constant, 2 Poisson)."""
    params = np.ascontiguousarray(params, dtype=dtype)
    n = params.shape[0]
    src = np.ascontiguousarray(src, dtype=np.int32)
    dst = np.ascontiguousarray(dst, dtype=np.int32)
    weight = np.ascontiguousarray(weight, dtype=dtype)
    delay_steps = np.ascontiguousarray(delay_steps, dtype=np.int32)
    s = src.shape[0]
    record_steps = min(record_steps, steps)
    if rec_ids is None:
        rec_ids = np.zeros(0, dtype=np.int32)
    rec_ids = np.ascontiguousarray(rec_ids, dtype=np.int32)
    if raster_cap is None:
        raster_cap = max(1, n * record_steps)
    fire_count = np.zeros(n, dtype=np.int32)
    raster_off = np.zeros(record_steps + 1, dtype=np.int64)
    raster_ids = np.zeros(raster_cap, dtype=np.int32)
    v_trace = np.zeros((record_steps, rec_ids.shape[0]), dtype=dtype)
    final_state = np.zeros((n, 4), dtype=dtype)
    spikes = np.zeros(steps, dtype=np.int64)
    events = np.zeros(steps, dtype=np.int64)
    if qexp is not None:
        qexp = np.ascontiguousarray(np.broadcast_to(np.asarray(qexp, dtype=np.int32), (n,)))
    if params_alt is not None:
        params_alt = np.ascontiguousarray(params_alt, dtype=dtype)
    if kind is not None:
        kind = np.ascontiguousarray(kind, dtype=np.uint8)
    if instance is not None:
        instance = np.ascontiguousarray(instance, dtype=np.int32)
    out = _Out(record_steps, _ptr(fire_count), _ptr(raster_off), _ptr(raster_ids), raster_cap,
               _ptr(rec_ids), rec_ids.shape[0], _ptr(v_trace), _ptr(final_state), _ptr(spikes),
               _ptr(events), _ptr(params_alt), int(half_period), _ptr(kind), _ptr(instance), int(input_seed))
    sfx = "f32" if dtype == np.float32 else "f64"
    rc = getattr(lib(), "oracle_run_" + sfx)(
        _ptr(params), n, _ptr(src), _ptr(dst), _ptr(weight), _ptr(delay_steps), s, dt, steps,
        acc_mode, _ptr(qexp), ctypes.byref(out))
    if rc != 0:
        raise RuntimeError("oracle_run failed with code %d" % rc)
    raster = [raster_ids[raster_off[t]:raster_off[t + 1]].copy() for t in range(record_steps)]
    return dict(fire_count=fire_count, raster=raster, v_trace=v_trace, final_state=final_state,
                spikes_per_step=spikes, events_per_step=events)


def poisson_draws(seed, rate, n):
    """n draws of the engine's Poisson sampler (draw i keyed as neuron i's first draw)."""
    out = np.zeros(n, dtype=np.int32)
    rc = lib().oracle_poisson_draws(int(seed), float(rate), int(n), _ptr(out))
    if rc != 0:
        raise RuntimeError("oracle_poisson_draws failed with code %d" % rc)
    return out


def ref_available(precision="f32"):
    return os.path.exists(os.path.join(REF_DIR, "ref_driver_" + precision))


def run_reference_many(net_path, copies, precision="f32"):
    """Runs `copies` instances of the reference's own simulator (oracle/_ref) on the
    same network file at once, one process each, without recording; returns each
    instance's loop time in seconds (its own timer)."""
    exe = os.path.join(REF_DIR, "ref_driver_" + precision)
    d = os.path.dirname(net_path)
    procs = []
    for k in range(copies):
        out = os.path.join(d, "out_%d.bin" % k)
        procs.append((out, subprocess.Popen([exe, net_path, out, "--no-record"], stdout=subprocess.DEVNULL)))
    secs = []
    for out, pr in procs:
        if pr.wait() != 0:
            raise RuntimeError("reference driver exited with %d" % pr.returncode)
        with open(out, "rb") as f:
            buf = f.read()
        secs.append(float(np.frombuffer(buf[-8:], dtype=np.float64)[0]))
    return secs


def run_reference(net_path, out_path, precision="f32", record=True, n=None, n_rec=0):
    """Run the reference's own simulator (oracle/_ref) on a network file written by
    tests/netio.write_net; parse its output file."""
    exe = os.path.join(REF_DIR, "ref_driver_" + precision)
    args = [exe, net_path, out_path] + ([] if record else ["--no-record"])
    subprocess.run(args, check=True, stdout=subprocess.DEVNULL)
    with open(out_path, "rb") as f:
        buf = f.read()
    pos = 0

    def take(dt, count):
        nonlocal pos
        a = np.frombuffer(buf, dtype=dt, count=count, offset=pos)
        pos += a.nbytes
        return a

    nrs = int(take(np.int64, 1)[0])
    counts = take(np.int64, nrs)
    nr = int(take(np.int64, 1)[0])
    ids = take(np.int32, nr)
    v = take(np.float64, nrs * n_rec).reshape(nrs, n_rec)
    fire_count = take(np.int32, n)
    last = take(np.float64, 5 * n).reshape(n, 5)
    secs = float(take(np.float64, 1)[0])
    offs = np.concatenate([[0], np.cumsum(counts)])
    raster = [ids[offs[t]:offs[t + 1]] for t in range(nrs)]
    return dict(raster=raster, v_trace=v, fire_count=fire_count, last_input=last, seconds=secs)


def gen_host(spec):
    """The seeded workload generator (the engine's own netgen.h, compiled into the oracle
    library): (params[n,10] f32, pop[n], src, dst, weight f32, delay_steps) in creation
    order, for a bsim_gen_spec, without loading the engine library."""
    L = lib()
    n, s = ctypes.c_int64(), ctypes.c_int64()
    if L.oracle_gen_count(ctypes.byref(spec), ctypes.byref(n), ctypes.byref(s)) != 0:
        raise ValueError("invalid generator spec")
    n, s = n.value, s.value
    params = np.zeros((n, 10), np.float32)
    pop = np.zeros(n, np.int32)
    src = np.zeros(s, np.int32)
    dst = np.zeros(s, np.int32)
    w = np.zeros(s, np.float32)
    d = np.zeros(s, np.int32)
    ptr = lambda a: ctypes.c_void_p(a.ctypes.data)
    if L.oracle_gen_host(ctypes.byref(spec), ptr(params), ptr(pop), ptr(src), ptr(dst), ptr(w), ptr(d)) != 0:
        raise ValueError("invalid generator spec")
    return dict(params=params, pop=pop, src=src, dst=dst, weight=w, delay_steps=d)
