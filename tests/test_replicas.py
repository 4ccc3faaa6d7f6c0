"""Several GPUs as replicas, host logic on CPU: two `gloo` ranks each simulate their own phonon
configurations (the FP64 oracle stands in for each rank's GPU), the patterns are summed with one
all-reduce, and the per-rank time is reduced to its maximum.  The summed pattern must equal the
sum of both ranks' patterns computed serially, and the ranks must draw different configurations."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _rank_main(rank, world, port, out_dir):
    sys.path.insert(0, ROOT)
    import datetime

    import torch
    import torch.distributed as dist

    from cudaem_b200 import replicas
    from cudaem_b200 import workloads as wl
    from oracle import oracle as orc
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        orc.set_threads(1)
        p, at = wl.cbed_si(cells=(2, 2, 2), n=128, nconf=1)
        q = replicas.for_rank(p, rank)
        pat = torch.from_numpy(np.ascontiguousarray(orc.simulate_cbed(q, at)))
        mine = pat.clone()
        replicas.sum_patterns(pat, dist)
        t = replicas.max_over_ranks(10.0 * (rank + 1), dist=dist)
        np.save(os.path.join(out_dir, f"r{rank}.npy"), mine.numpy())
        np.save(os.path.join(out_dir, f"sum{rank}.npy"), pat.numpy())
        np.save(os.path.join(out_dir, f"t{rank}.npy"), np.array([t, replicas.mean_weight(dist)]))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks(tmp_path):
    import socket

    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    r0, r1 = np.load(tmp_path / "r0.npy"), np.load(tmp_path / "r1.npy")
    assert not np.allclose(r0, r1)                       # different phonon configurations
    for k in (0, 1):
        assert np.allclose(np.load(tmp_path / f"sum{k}.npy"), r0 + r1, rtol=1e-12, atol=0)
        t, w = np.load(tmp_path / f"t{k}.npy")
        assert t == 20.0 and w == 0.5


def test_rank_seeds():
    from cudaem_b200 import replicas
    from cudaem_b200 import workloads as wl
    p, _ = wl.cbed_si(cells=(2, 2, 2), n=128, nconf=1)
    seeds = {replicas.for_rank(p, r).pn_seed for r in range(8)}
    assert len(seeds) == 8 and replicas.for_rank(p, 0).pn_seed == p.pn_seed
