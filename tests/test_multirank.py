"""The N > 1 host logic (phcpack_b200.multirank) with world size 2 on CPU:
gloo processes split the paths of a homotopy into shards, track them (the
CPU tracker of the oracle stands in for the GPU here), take the maximum of
their times and gather the per-path results on rank 0, which must equal one
process tracking everything."""
import os
import socket

import numpy as np
import pytest

from phcpack_b200 import multirank


def test_shard_covers_units_once():
    for n in (0, 1, 7, 1024, 1025):
        for world in (1, 2, 3, 8):
            got = [u for r in range(world) for u in multirank.shard(n, r, world)]
            assert got == list(range(n))
            sizes = [len(multirank.shard(n, r, world)) for r in range(world)]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        multirank.shard(10, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_path):
    import datetime
    import time
    import torch.distributed as dist
    from oracle import pyoracle
    from phcpack_b200 import homotopy as hm
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    pb = hm.subset(hm.config4(), np.arange(0, 1024, 64))
    mine = multirank.shard(pb.npaths, rank, world)
    sub = hm.subset(pb, np.arange(mine.start, mine.stop))
    ipar, dpar = hm.params()
    dist.barrier()
    t = time.perf_counter()
    xend, info, dinfo = pyoracle.track(pyoracle.oracle(), sub, ipar, dpar, pmode=1, rmode=2)
    elapsed = time.perf_counter() - t
    tmax = multirank.max_over_ranks(elapsed, dist)
    rows = np.concatenate([info.reshape(-1, 6).astype(np.float64), dinfo.reshape(-1, 2),
                           xend.reshape(len(mine), -1)], axis=1)
    allrows = multirank.gather_rows(rows, pb.npaths, dist)
    if rank == 0:
        np.savez(out_path, rows=allrows, tmax=tmax, mine=elapsed)
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_track_shards_and_gather(tmp_path):
    import torch.multiprocessing as mp
    from oracle import pyoracle
    from phcpack_b200 import homotopy as hm
    out = str(tmp_path / "r.npz")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    d = np.load(out)
    pb = hm.subset(hm.config4(), np.arange(0, 1024, 64))
    ipar, dpar = hm.params()
    xend, info, dinfo = pyoracle.track(pyoracle.oracle(), pb, ipar, dpar, pmode=1, rmode=2)
    one = np.concatenate([info.reshape(-1, 6).astype(np.float64), dinfo.reshape(-1, 2),
                          xend.reshape(pb.npaths, -1)], axis=1)
    assert np.array_equal(d["rows"], one)  # same per-path results, in path order
    assert float(d["tmax"]) >= float(d["mine"])
