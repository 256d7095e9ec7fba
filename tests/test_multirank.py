"""bench.py's multi-GPU path runs one independent network per rank and combines
the ranks' numbers with one max and one sum reduction; this checks that
combination with two gloo ranks on the CPU (no GPU involved)."""
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
