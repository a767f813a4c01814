"""The N-GPU path of bench.py without GPUs: two ranks over gloo (127.0.0.1) run the same
barrier and max-over-ranks reduction the bench uses around its timed region, and the
whole-job value is computed from the slowest rank."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench

    d = bench.Dist(backend="gloo")
    d.barrier()
    ms = 10.0 + 5.0 * rank  # the slower rank decides
    ms_max = d.max(ms)
    d.barrier()
    out[rank] = (d.rank, d.world, ms_max, bench.aggregate_value(d.world, 1000, 4, ms_max))
    d.close()


def test_two_ranks_take_the_maximum_time():
    world, port = 2, _free_port()
    with mp.Manager() as man:
        out = man.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert sorted(res) == [0, 1]
    for r, (rank, w, ms_max, value) in res.items():
        assert rank == r and w == world and ms_max == 15.0
        assert value == pytest.approx(world * 1000 * 4 / 15e-3)
