"""bench.py's multi-GPU path runs one independent network per rank and combines
the ranks' numbers with one max and one sum reduction; this checks that
combination with two gloo ranks on the CPU (no GPU involved), and that a rank
which leaves makes the others' next reduction fail instead of hang."""
import os
import socket

import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = [10.0, 12.5][rank]
    events = [1000, 3000][rank]
    (ms_max,), (ev_sum, n_sum) = bench.reduce_over_ranks(dist, [ms], [events, 5])
    out[rank] = (ms_max, ev_sum, n_sum)
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_max_time_and_sum_events():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    for r in (0, 1):
        assert res[r] == (12.5, 4000.0, 10.0)
    # weak scaling: whole-job events/s = all ranks' events over the slowest rank's time
    assert res[0][1] / (res[0][0] / 1e3) == 4000 / 0.0125


def test_single_process_passthrough():
    assert bench.reduce_over_ranks(None, [1.5], [2, 3]) == ([1.5], [2.0, 3.0])


def _rank_leaves(rank, world, port, out):
    import datetime
    import time
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    if rank == 1:
        os._exit(3)  # leaves between steps, with no collective in flight
    t0 = time.time()
    try:
        bench.reduce_over_ranks(dist, [1.0], [1])
        out[rank] = ("no error", time.time() - t0)
    except Exception as ex:  # the peer's departure surfaces as an error, not a hang
        out[rank] = (type(ex).__name__, time.time() - t0)


def test_a_rank_that_leaves_ends_the_others_reduction_with_an_error():
    """Failure detection on the host: one rank exits after joining; the other's
    next reduction raises within the process group's timeout instead of hanging."""
    ctx = mp.get_context("spawn")
    port = _free_port()
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_rank_leaves, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        alive = [p for p in procs if p.is_alive()]
        for p in alive:
            p.kill()
        res = dict(out)
    assert not alive
    assert procs[1].exitcode == 3
    kind, waited = res[0]
    assert kind != "no error" and waited < 60.0
