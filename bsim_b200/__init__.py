"""Python binding of the bsim_b200 C ABI (include/bsim_b200.h).

The engine is the CUDA library libbsim_b200.so built in this directory
(bsim_b200/build.py). There is no CPU fallback: if the library is missing or a
call fails, an exception is raised.

Mirrors the reference's SGSim path: an Engine is what SingleGPUSimulator::run
builds (src/sim/SingleGPUSimulator.cu:31-144); Engine.run(steps) is its step
loop (:146-245); fire_count() is FireInfo "count" (:263-282).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbsim_b200.so")

BSIM_OK = 0
ACC_EXACT = 0
ACC_ORDERED = 1
DELIVERY_PUSH = 0
DELIVERY_PULL = 1
DELIVERY_AUTO = 2
DELIVERY_TILE = 3
NEURON_LIF = 0
NEURON_CONSTANT = 1
NEURON_POISSON = 2
MAX_DELAY = 1024


class BsimError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("bsim error %d: %s" % (code, msg))
        self.code = code


class Options(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("accumulate", ctypes.c_int32), ("delivery", ctypes.c_int32),
                ("build_pull", ctypes.c_int32), ("graph_steps", ctypes.c_int32),
                ("block_threads", ctypes.c_int32), ("grid_blocks", ctypes.c_int32),
                ("build_tiles", ctypes.c_int32), ("tile_size", ctypes.c_int32),
                ("reserved", ctypes.c_int32 * 7)]


class GenSpec(ctypes.Structure):
    _fields_ = [("seed", ctypes.c_uint64), ("n_pop", ctypes.c_int32), ("pop_size", ctypes.c_int32),
                ("p_conn", ctypes.c_float), ("remote_frac", ctypes.c_float), ("max_delay", ctypes.c_int32),
                ("exc_frac", ctypes.c_float), ("w_max", ctypes.c_float), ("inh_scale", ctypes.c_float),
                ("i_min", ctypes.c_float), ("i_max", ctypes.c_float),
                ("v_init_lo", ctypes.c_float), ("v_init_hi", ctypes.c_float),
                ("v_rest", ctypes.c_float), ("v_reset", ctypes.c_float), ("cm", ctypes.c_float),
                ("tau_m", ctypes.c_float), ("tau_refrac", ctypes.c_float), ("tau_syn_E", ctypes.c_float),
                ("tau_syn_I", ctypes.c_float), ("v_thresh", ctypes.c_float),
                ("drive_scale", ctypes.c_float), ("drive_half_period", ctypes.c_int32)]


class Info(ctypes.Structure):
    _fields_ = [("n_neurons", ctypes.c_int64), ("n_synapses", ctypes.c_int64), ("max_delay", ctypes.c_int32),
                ("n_instances", ctypes.c_int32), ("n_classes", ctypes.c_int32), ("n_pops", ctypes.c_int32),
                ("steps_done", ctypes.c_int64), ("events_total", ctypes.c_uint64),
                ("device_bytes", ctypes.c_int64), ("grid_blocks", ctypes.c_int32),
                ("block_threads", ctypes.c_int32), ("accumulate", ctypes.c_int32),
                ("delivery", ctypes.c_int32), ("sm_count", ctypes.c_int32), ("reserved", ctypes.c_int32 * 7)]


EXPORTS = [
    "bsim_options_default", "bsim_create", "bsim_create_mixed", "bsim_create_generated", "bsim_gen_count", "bsim_gen_host",
    "bsim_synapse_reset", "bsim_run", "bsim_run_async", "bsim_sync", "bsim_record", "bsim_read_raster",
    "bsim_read_state", "bsim_read_fire_count", "bsim_read_pop_counts", "bsim_get_info", "bsim_get_qexp",
    "bsim_destroy", "bsim_last_error", "bsim_write_state", "bsim_get_stream", "bsim_set_drive",
    "bsim_enable_pop_stats", "bsim_read_pop_info", "bsim_mlp_init", "bsim_mlp_forward", "bsim_mlp_grad",
    "bsim_mlp_train", "bsim_set_predictor", "bsim_predictor_stats", "bsim_autotune", "bsim_stall_tile",
]

MLP_IN = 9
MLP_HIDDEN = 64
MLP_PARAMS = MLP_HIDDEN * MLP_IN + MLP_HIDDEN + MLP_HIDDEN * MLP_HIDDEN + MLP_HIDDEN + MLP_HIDDEN + 1


class PredStats(ctypes.Structure):
    _fields_ = [("cycles", ctypes.c_int64), ("fallbacks", ctypes.c_int64), ("tile_cycles", ctypes.c_int64),
                ("abs_err_sum", ctypes.c_double), ("actual_sum", ctypes.c_double)]


class TuneResult(ctypes.Structure):
    _fields_ = [("block_threads", ctypes.c_int32), ("grid_blocks", ctypes.c_int32), ("delivery", ctypes.c_int32),
                ("best_us_per_step", ctypes.c_float), ("cost_push", ctypes.c_float * 2),
                ("cost_tile", ctypes.c_float * 2), ("candidates", ctypes.c_int32)]

_lib = None


def lib():
    """Loads libbsim_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("bsim_b200: %s is missing; build it with `python -m bsim_b200.build`" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        i32, i64, f32 = ctypes.c_int32, ctypes.c_int64, ctypes.c_float
        sig = {
            "bsim_options_default": [P],
            "bsim_create": [P, i64, P, P, P, P, P, P, i64, f32, P, P],
            "bsim_create_mixed": [P, P, i64, P, P, P, P, P, P, i64, f32, ctypes.c_uint64, P, P],
            "bsim_create_generated": [P, i32, f32, P, P],
            "bsim_gen_count": [P, P, P],
            "bsim_gen_host": [P, P, P, P, P, P, P],
            "bsim_synapse_reset": [P, P, P, i64, f32, P, P],
            "bsim_run": [P, i64],
            "bsim_run_async": [P, i64],
            "bsim_sync": [P],
            "bsim_stall_tile": [P, i32],
            "bsim_record": [P, i64, i64],
            "bsim_read_raster": [P, P, P, i64, P],
            "bsim_read_state": [P, P, P, P, P],
            "bsim_read_fire_count": [P, P],
            "bsim_read_pop_counts": [P, P, i32],
            "bsim_get_info": [P, P],
            "bsim_get_qexp": [P, P],
            "bsim_destroy": [P],
            "bsim_write_state": [P, P, P, P, P],
            "bsim_get_stream": [P, P],
            "bsim_set_drive": [P, P, i32],
            "bsim_enable_pop_stats": [P, i32],
            "bsim_read_pop_info": [P, P, P, P],
            "bsim_mlp_init": [P, ctypes.c_uint64],
            "bsim_mlp_forward": [P, P, i64, P],
            "bsim_mlp_grad": [P, P, P, i64, P, P],
            "bsim_mlp_train": [P, P, P, i64, i32, i32, f32, ctypes.c_uint64, P],
            "bsim_set_predictor": [P, P, f32, P, P],
            "bsim_predictor_stats": [P, P],
            "bsim_autotune": [P, i32, P],
            "bsim_trace": [P, i64, i64, i64],
            "bsim_read_trace": [P, P, P, P, P, P, P],
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = ctypes.c_int
        L.bsim_last_error.argtypes = []
        L.bsim_last_error.restype = ctypes.c_char_p
        _lib = L
    return _lib


def _check(rc):
    if rc != BSIM_OK:
        raise BsimError(rc, lib().bsim_last_error().decode(errors="replace"))


def _p(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def options(**kw):
    o = Options()
    _check(lib().bsim_options_default(ctypes.byref(o)))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def gen_spec(**kw):
    """A generated-network spec with the LIF_brian defaults of the CUBA workload
    (v_rest = v_reset = -65 mV, v_thresh = -50 mV, cm = 0.25 nF, tau_m = 20 ms,
    tau_refrac = 2 ms, tau_syn_E = 5 ms, tau_syn_I = 10 ms, p = 0.1, 20 % remote,
    80 % excitatory, inhibitory weights 4x)."""
    d = dict(seed=1, n_pop=10, pop_size=1000, p_conn=0.1, remote_frac=0.2, max_delay=6, exc_frac=0.8,
             w_max=1e-10, inh_scale=4.0, i_min=0.0, i_max=1.1e-9, v_init_lo=-65e-3, v_init_hi=-50e-3,
             v_rest=-65e-3, v_reset=-65e-3, cm=0.25e-9, tau_m=20e-3, tau_refrac=2e-3, tau_syn_E=5e-3,
             tau_syn_I=10e-3, v_thresh=-50e-3, drive_scale=1.0, drive_half_period=0)
    d.update(kw)
    s = GenSpec()
    for k, v in d.items():
        setattr(s, k, v)
    return s


def gen_host(spec):
    """Host generator: (params[n,10] f32, pop[n], src, dst, weight f32, delay_steps) in creation order."""
    n = ctypes.c_int64()
    s = ctypes.c_int64()
    _check(lib().bsim_gen_count(ctypes.byref(spec), ctypes.byref(n), ctypes.byref(s)))
    n, s = n.value, s.value
    params = np.zeros((n, 10), np.float32)
    pop = np.zeros(n, np.int32)
    src = np.zeros(s, np.int32)
    dst = np.zeros(s, np.int32)
    w = np.zeros(s, np.float32)
    d = np.zeros(s, np.int32)
    _check(lib().bsim_gen_host(ctypes.byref(spec), _p(params), _p(pop), _p(src), _p(dst), _p(w), _p(d)))
    return dict(params=params, pop=pop, src=src, dst=dst, weight=w, delay_steps=d)


def mlp_init(seed=1):
    p = np.zeros(MLP_PARAMS, np.float32)
    _check(lib().bsim_mlp_init(_p(p), seed))
    return p


def mlp_forward(params, x):
    params = np.ascontiguousarray(params, np.float32)
    x = np.ascontiguousarray(x, np.float32)
    y = np.zeros(x.shape[0], np.float32)
    _check(lib().bsim_mlp_forward(_p(params), _p(x), x.shape[0], _p(y)))
    return y


def mlp_grad(params, x, y):
    params = np.ascontiguousarray(params, np.float32)
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    g = np.zeros(MLP_PARAMS, np.float32)
    loss = ctypes.c_float()
    _check(lib().bsim_mlp_grad(_p(params), _p(x), _p(y), x.shape[0], _p(g), ctypes.byref(loss)))
    return g, loss.value


def mlp_train(params, x, y, epochs=20, batch=256, lr=1e-3, seed=1):
    params = np.array(params, np.float32)
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    loss = ctypes.c_float()
    _check(lib().bsim_mlp_train(_p(params), _p(x), _p(y), x.shape[0], epochs, batch, lr, seed, ctypes.byref(loss)))
    return params, loss.value


def synapse_reset(delay_s, weight, tau_syn, dt):
    d = np.ascontiguousarray(delay_s, np.float32)
    w = np.ascontiguousarray(weight, np.float32)
    t = np.ascontiguousarray(tau_syn, np.float32)
    st = np.zeros(d.shape[0], np.int32)
    wo = np.zeros(d.shape[0], np.float32)
    _check(lib().bsim_synapse_reset(_p(d), _p(w), _p(t), d.shape[0], dt, _p(st), _p(wo)))
    return st, wo


class Engine:
    """One engine: one or more independent networks on one GPU."""

    def __init__(self, handle):
        self._h = handle
        self._rec_steps = None  # steps of the current recording (sizes the offsets read back)

    @classmethod
    def from_arrays(cls, params, src, dst, weight, delay_steps, dt, pop=None, instance=None, opts=None,
                    kind=None, input_seed=0):
        """kind: per-neuron NEURON_LIF / NEURON_CONSTANT / NEURON_POISSON (None: all LIF);
        input_seed: seed of the Poisson neurons' draws."""
        params = np.ascontiguousarray(params, np.float32)
        src = np.ascontiguousarray(src, np.int32)
        dst = np.ascontiguousarray(dst, np.int32)
        weight = np.ascontiguousarray(weight, np.float32)
        delay_steps = np.ascontiguousarray(delay_steps, np.int32)
        pop = None if pop is None else np.ascontiguousarray(pop, np.int32)
        instance = None if instance is None else np.ascontiguousarray(instance, np.int32)
        opts = opts or options()
        h = ctypes.c_void_p()
        if kind is None:
            _check(lib().bsim_create(_p(params), params.shape[0], _p(pop), _p(instance), _p(src), _p(dst),
                                     _p(weight), _p(delay_steps), src.shape[0], dt, ctypes.byref(opts),
                                     ctypes.byref(h)))
        else:
            kind = np.ascontiguousarray(kind, np.uint8)
            _check(lib().bsim_create_mixed(_p(params), _p(kind), params.shape[0], _p(pop), _p(instance), _p(src),
                                           _p(dst), _p(weight), _p(delay_steps), src.shape[0], dt, input_seed,
                                           ctypes.byref(opts), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def generated(cls, specs, dt, opts=None):
        if isinstance(specs, GenSpec):
            specs = [specs]
        arr = (GenSpec * len(specs))(*specs)
        opts = opts or options()
        h = ctypes.c_void_p()
        _check(lib().bsim_create_generated(arr, len(specs), dt, ctypes.byref(opts), ctypes.byref(h)))
        return cls(h)

    def run(self, steps):
        _check(lib().bsim_run(self._h, steps))

    def run_async(self, steps):
        _check(lib().bsim_run_async(self._h, steps))

    def sync(self):
        _check(lib().bsim_sync(self._h))

    def record(self, max_steps, capacity):
        _check(lib().bsim_record(self._h, max_steps, capacity))
        self._rec_steps = max_steps

    def raster(self, out=None):
        """Recorded spikes: list of int32 arrays (ascending ids), one per recorded step.
        The arrays are views into one buffer read in a single copy from the device:
        `out` (a C-contiguous int32 array, e.g. in page-locked memory, reused across
        reads) when it is large enough, else a new array."""
        if self._rec_steps is None:
            self._rec_steps = self.info().steps_done + 1
        off = np.zeros(self._rec_steps + 2, np.int64)
        ns = ctypes.c_int64()
        if out is not None and out.dtype == np.int32 and out.ndim == 1 and out.flags.c_contiguous:
            # one call: sizes and ids together when `out` is large enough
            rc = lib().bsim_read_raster(self._h, _p(off), _p(out), out.shape[0], ctypes.byref(ns))
            if rc == BSIM_OK:
                return [out[off[k]:off[k + 1]] for k in range(ns.value)]
        _check(lib().bsim_read_raster(self._h, _p(off), None, 0, ctypes.byref(ns)))
        total = int(off[ns.value])
        if (out is not None and out.dtype == np.int32 and out.ndim == 1 and out.flags.c_contiguous
                and out.shape[0] >= max(total, 1)):
            ids = out
        else:
            ids = np.empty(max(total, 1), np.int32)
        _check(lib().bsim_read_raster(self._h, _p(off), _p(ids), ids.shape[0], ctypes.byref(ns)))
        return [ids[off[k]:off[k + 1]] for k in range(ns.value)]

    def trace(self, max_steps, first=0, count=None):
        """Traces v, i_E, i_I and the consumed synaptic input (E, I) of neurons
        [first, first + count) after each of the next max_steps cycles, on the device."""
        if count is None:
            count = self.info().n_neurons - first
        _check(lib().bsim_trace(self._h, max_steps, first, count))
        self._trace_shape = (max_steps, count)

    def read_trace(self):
        """The trace so far: dict of [n_steps, count] float32 arrays v, i_E, i_I, in_E, in_I."""
        steps, count = self._trace_shape
        out = {k: np.zeros((steps, count), np.float32) for k in ("v", "i_E", "i_I", "in_E", "in_I")}
        ns = ctypes.c_int64()
        _check(lib().bsim_read_trace(self._h, _p(out["v"]), _p(out["i_E"]), _p(out["i_I"]), _p(out["in_E"]),
                                     _p(out["in_I"]), ctypes.byref(ns)))
        return {k: v[:ns.value] for k, v in out.items()}

    def state(self):
        n = self.info().n_neurons
        v = np.zeros(n, np.float32)
        ie = np.zeros(n, np.float32)
        ii = np.zeros(n, np.float32)
        rf = np.zeros(n, np.int32)
        _check(lib().bsim_read_state(self._h, _p(v), _p(ie), _p(ii), _p(rf)))
        return dict(v=v, i_E=ie, i_I=ii, refrac=rf)

    def write_state(self, v=None, i_E=None, i_I=None, refrac=None):
        c = lambda a, t: None if a is None else np.ascontiguousarray(a, t)
        v, i_E, i_I, refrac = c(v, np.float32), c(i_E, np.float32), c(i_I, np.float32), c(refrac, np.int32)
        _check(lib().bsim_write_state(self._h, _p(v), _p(i_E), _p(i_I), _p(refrac)))

    def set_drive(self, params_hi, half_period):
        p = np.ascontiguousarray(params_hi, np.float32)
        _check(lib().bsim_set_drive(self._h, _p(p), half_period))

    def enable_pop_stats(self, hist_len=64):
        _check(lib().bsim_enable_pop_stats(self._h, hist_len))

    def pop_counts(self, steps):
        P = self.info().n_pops
        c = np.zeros((steps, P), np.int32)
        _check(lib().bsim_read_pop_counts(self._h, _p(c), steps))
        return c

    def pop_info(self):
        P = self.info().n_pops
        size = np.zeros(P, np.int32)
        ind = np.zeros(P, np.float32)
        outd = np.zeros(P, np.float32)
        _check(lib().bsim_read_pop_info(self._h, _p(size), _p(ind), _p(outd)))
        return size, ind, outd

    def set_predictor(self, params, tolerance=0.25, cost_push=None, cost_tile=None):
        cp = None if cost_push is None else np.ascontiguousarray(cost_push, np.float32)
        ct = None if cost_tile is None else np.ascontiguousarray(cost_tile, np.float32)
        pp = None if params is None else np.ascontiguousarray(params, np.float32)
        _check(lib().bsim_set_predictor(self._h, _p(pp), tolerance, _p(cp), _p(ct)))

    def predictor_stats(self):
        st = PredStats()
        _check(lib().bsim_predictor_stats(self._h, ctypes.byref(st)))
        return st

    def autotune(self, trial_steps=50):
        r = TuneResult()
        _check(lib().bsim_autotune(self._h, trial_steps, ctypes.byref(r)))
        return r

    def stream(self):
        """The engine's cudaStream_t as an integer handle (for torch.cuda.ExternalStream)."""
        s = ctypes.c_void_p()
        _check(lib().bsim_get_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    def fire_count(self, out=None):
        """Spikes per neuron since creation; into `out` (a C-contiguous int32 array of
        n_neurons, e.g. in page-locked memory, reused across reads) when given."""
        n = self.info().n_neurons
        if (out is not None and out.dtype == np.int32 and out.ndim == 1 and out.flags.c_contiguous
                and out.shape[0] == n):
            c = out
        else:
            c = np.zeros(n, np.int32)
        _check(lib().bsim_read_fire_count(self._h, _p(c)))
        return c

    def info(self):
        i = Info()
        _check(lib().bsim_get_info(self._h, ctypes.byref(i)))
        return i

    def qexp(self):
        q = np.zeros(self.info().n_instances, np.int32)
        _check(lib().bsim_get_qexp(self._h, _p(q)))
        return q

    def close(self):
        if self._h:
            lib().bsim_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
