"""The multi-rank path on CPU: two gloo ranks (spawned processes) shard points
contiguously, evaluate their own slices (the oracle's field stands in for the
GPU kernel here), gather, and take the max of a per-rank timing -- the same
functions bench.py and multi-GPU callers use over NCCL."""
import os
import socket
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world_size, port, out_dir):
    sys.path.insert(0, os.path.join(ROOT, "c-coil_b200"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import torch.distributed as dist
    from ccoil_b200 import distributed as D
    from ccoil_b200 import workloads
    from oracle import Oracle
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world_size)
    try:
        O = Oracle()
        rows, pts = workloads.group_config(coils=3, points=101)
        full = D.evaluate_sharded(lambda p: O.group_fields(rows, p, 1, pf=3.0), pts)
        lo, hi, local = D.evaluate_sharded(lambda p: O.group_fields(rows, p, 1, pf=3.0), pts, gather=False)
        mx = D.max_over_ranks(1.5 + rank)
        D.barrier()
        np.savez(os.path.join(out_dir, "rank%d.npz" % rank), full=full.numpy(), lo=lo, hi=hi,
                 local=local.numpy(), mx=mx, world=D.world()[1])
    finally:
        dist.destroy_process_group()


def test_shard_bounds_cover_exactly():
    sys.path.insert(0, os.path.join(ROOT, "c-coil_b200"))
    from ccoil_b200.distributed import shard_bounds
    for n in (0, 1, 7, 100, 1 << 20):
        for w in (1, 2, 3, 8):
            bounds = [shard_bounds(n, r, w) for r in range(w)]
            assert bounds[0][0] == 0 and bounds[-1][1] == n
            assert all(bounds[i][1] == bounds[i + 1][0] for i in range(w - 1))
            sizes = [hi - lo for lo, hi in bounds]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_bounds(10, 2, 2)


def test_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "c-coil_b200"))
    from oracle import Oracle
    from ccoil_b200 import workloads
    mp.spawn(_rank_main, args=(2, free_port(), str(tmp_path)), nprocs=2, join=True)
    rows, pts = workloads.group_config(coils=3, points=101)
    ref = Oracle().group_fields(rows, pts, 1, pf=3.0)
    got = [np.load(os.path.join(tmp_path, "rank%d.npz" % r)) for r in range(2)]
    for r, g in enumerate(got):
        assert int(g["world"]) == 2
        assert float(g["mx"]) == 2.5                       # max over ranks of 1.5 + rank
        assert np.array_equal(g["full"], ref)              # slices gathered in rank order
        lo, hi = int(g["lo"]), int(g["hi"])
        assert (lo, hi) == ((0, 51) if r == 0 else (51, 101))
        assert np.array_equal(g["local"], ref[lo:hi])
