"""The allocation-free step (bsim_run_noalloc), for callers that cannot allocate
device memory: the test plays such a caller. It owns every buffer (allocated
here with torch, as a host application's pool would), passes device pointers
through the C ABI, and checks the result against the regular engine
(bsim_create + bsim_run) on the same network. Bit-identical is the bar, as for
the other EXACT-mode comparisons. Several calls run in a row on different
networks, so a call that inherited the previous call's working memory would
show up as a mismatch."""
import ctypes

import numpy as np
import pytest

import bsim_b200 as B
from bsim_b200 import workloads as W
from oracle import oracle

pytestmark = pytest.mark.gpu
DT = np.float32(1e-4)

CLASS_DTYPE = np.dtype([("Cm", "<f4"), ("CE", "<f4"), ("CI", "<f4"), ("C_E", "<f4"), ("C_I", "<f4"),
                        ("v_thresh", "<f4"), ("v_reset", "<f4"), ("refrac_time", "<i4"), ("scale_up", "<f4"),
                        ("scale_down", "<f4"), ("pop", "<i4"), ("inst", "<i4"), ("kind", "<i4"),
                        ("id_base", "<i4"), ("reserved", "<i4", (2,))])


def noalloc_fn():
    f = B.lib().bsim_run_noalloc
    P = ctypes.c_void_p
    f.argtypes = [ctypes.c_int64, ctypes.c_int32, P, P, P, P, ctypes.c_int32, P, P, ctypes.c_int64, P,
                  ctypes.c_int64, P]
    f.restype = ctypes.c_int
    return f


def status(stream):
    """The device error flag of the last call (bsim_noalloc_status): (return code, flag)."""
    f = B.lib().bsim_noalloc_status
    f.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32)]
    f.restype = ctypes.c_int
    err = ctypes.c_int32(-1)
    rc = f(stream, ctypes.byref(err))
    return rc, err.value


def caller_buffers(g, qexp, D):
    """The inputs a caller hands over, in the layout bsim_b200.h documents, as torch device tensors."""
    import torch
    params = g["params"]
    n = params.shape[0]
    fold, rt = oracle.lif_reset(params, DT)  # LIFENeuron::reset, fp32
    pops = g["pop"]
    P = int(pops.max()) + 1
    ctab = np.zeros(P, CLASS_DTYPE)
    for p in range(P):
        i = int(np.flatnonzero(pops == p)[0])
        ctab[p] = (fold[i, 10], fold[i, 2], fold[i, 1], fold[i, 4], fold[i, 3], fold[i, 8], fold[i, 9], rt[i],
                   np.ldexp(np.float32(1), qexp), np.ldexp(np.float32(1), -qexp), p, 0, 0, 0, (0, 0))
    state = np.zeros((n, 4), np.float32)
    state[:, 0] = params[:, 0]
    key = g["src"].astype(np.int64) * D + (g["delay_steps"] - 1)
    order = np.argsort(key, kind="stable")
    row_off = np.zeros(n * D + 1, np.int64)
    row_off[1:] = np.cumsum(np.bincount(key, minlength=n * D))
    # {target, weight bits} pairs, held as int32 (the same bits; torch indexes int32 tensors)
    syn = np.stack([g["dst"].astype(np.int32)[order], g["weight"].view(np.int32)[order]], 1)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return dict(state=dev(state), vtmp=dev(fold[:, 5].copy()), cls=dev(pops.astype(np.int16)),
                ctab=dev(ctab.view(np.uint8)), row_off=dev(row_off), syn=dev(syn),
                fire_count=dev(np.zeros(n, np.int32)))


def run_noalloc(fn, bufs, n, D, steps, expect_ok=True):
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    n_cls = bufs["ctab"].numel() // CLASS_DTYPE.itemsize
    rc = fn(n, D, bufs["state"].data_ptr(), bufs["vtmp"].data_ptr(), bufs["cls"].data_ptr(), bufs["ctab"].data_ptr(),
            n_cls, bufs["row_off"].data_ptr(), bufs["syn"].data_ptr(), bufs["syn"].shape[0],
            bufs["fire_count"].data_ptr(), steps, stream)
    assert rc == 0, B.lib().bsim_last_error()
    src, flag = status(stream)
    if expect_ok:
        assert src == 0 and flag == 0, B.lib().bsim_last_error()
    torch.cuda.synchronize()
    st = bufs["state"].cpu().numpy()
    return st[:, 0].copy(), st[:, 1].copy(), st[:, 2].copy(), st[:, 3].view(np.int32).copy(), \
        bufs["fire_count"].cpu().numpy(), flag


def run_engine(g, steps):
    eng = B.Engine.from_arrays(g["params"], g["src"], g["dst"], g["weight"], g["delay_steps"], DT, pop=g["pop"])
    eng.run(steps)
    s = eng.state()
    out = (s["v"], s["i_E"], s["i_I"], s["refrac"], eng.fire_count(), int(eng.qexp()[0]))
    eng.close()
    return out


def check_against_engine(fn, spec, steps):
    g = B.gen_host(spec)
    n = g["params"].shape[0]
    ref = run_engine(g, steps)
    bufs = caller_buffers(g, ref[5], spec.max_delay)
    got = run_noalloc(fn, bufs, n, spec.max_delay, steps)
    assert ref[4].sum() > 0
    for a, b in zip(got[:5], ref[:5]):
        assert np.array_equal(a, b)


def test_noalloc_matches_engine_on_consecutive_calls():
    fn = noalloc_fn()
    nets = [(W.cuba(10, 1000, 100, 6, seed=31), 300),
            (W.cuba(8, 600, 500, 12, seed=32), 200),
            (W.cuba(10, 1000, 100, 6, seed=31), 300)]
    for spec, steps in nets:
        check_against_engine(fn, spec, steps)


def test_noalloc_at_its_size_limits():
    """n = BSIM_NOALLOC_MAX_NEURONS with max_delay = BSIM_NOALLOC_MAX_DELAY: the ring
    region of the array is full, so an off-by-one in the array's layout would show."""
    fn = noalloc_fn()
    for spec, steps in ((W.cuba(16, 2048, 100, 16, seed=33), 150), (W.cuba(16, 2048, 500, 16, seed=34), 150)):
        assert spec.n_pop * spec.pop_size == 32768 and spec.max_delay == 16
        check_against_engine(fn, spec, steps)


def test_noalloc_flags_corrupt_inputs_without_running_them():
    """Corrupted caller arrays (a target outside the network, descending row
    offsets, offsets that do not end at the synapse count, a class index beyond
    the table, a class of another kind) are caught by the check pass on the GPU:
    bsim_noalloc_status reports the code and no cycle ran (state and counts
    unchanged). Every access stays inside the arrays, so nothing faults. The next
    valid call starts clean."""
    import torch
    fn = noalloc_fn()
    spec = W.cuba(4, 500, 500, 6, seed=35)
    g = B.gen_host(spec)
    n = g["params"].shape[0]
    ref = run_engine(g, 50)
    good = caller_buffers(g, ref[5], spec.max_delay)

    def corrupted(what):
        b = {k: v.clone() for k, v in good.items()}
        if what == "target":
            b["syn"][len(b["syn"]) // 2, 0] = n + 5
        elif what == "row":
            k = int(torch.nonzero(b["row_off"][1:] > b["row_off"][:-1])[5])
            b["row_off"][k + 1] = b["row_off"][k] - 1
        elif what == "rows_end":
            b["row_off"][-1] += 2  # still ascending, but past the synapse count
        elif what == "class":
            b["cls"][7] = 4  # 4 classes (one per population): 4 is past the table
        elif what == "kind":
            ct = b["ctab"].cpu().numpy().view(CLASS_DTYPE).copy()
            ct["kind"][2] = 2
            b["ctab"] = torch.from_numpy(ct.view(np.uint8)).cuda()
        return b

    codes = {"row": 1, "target": 2, "class": 3, "kind": 3, "rows_end": 4}
    for what, code in codes.items():
        b = corrupted(what)
        st0 = b["state"].cpu().numpy().copy()
        got = run_noalloc(fn, b, n, spec.max_delay, 50, expect_ok=False)
        assert got[5] == code, (what, got[5])
        assert np.array_equal(b["state"].cpu().numpy(), st0)
        assert got[4].sum() == 0
        assert status(torch.cuda.current_stream().cuda_stream)[0] == -3  # BSIM_ERR_DEVICE
    got = run_noalloc(fn, good, n, spec.max_delay, 50)
    for a, b in zip(got[:5], ref[:5]):
        assert np.array_equal(a, b)


def test_noalloc_rejects_sizes_beyond_its_array():
    """Sizes beyond the array are refused before any pointer is used or any work is enqueued."""
    fn = noalloc_fn()
    assert fn(32769, 6, 16, 16, 16, 16, 1, 16, 16, 0, 16, 1, None) == -7  # BSIM_ERR_LIMIT
    assert "32768" in B.lib().bsim_last_error().decode()
    assert fn(100, 17, 16, 16, 16, 16, 1, 16, 16, 0, 16, 1, None) == -7
