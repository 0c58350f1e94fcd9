"""Frequency sharding over ranks, as bench.py and a multi-GPU deck run use it,
exercised with two gloo ranks on the CPU: each rank solves its contiguous
block of the frequencies with the CPU oracle, rank 0 gathers the results in
frequency order, and they equal a single-process run bit for bit; the
max-over-ranks of a timing is the slowest rank's.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "hams-mrel_b200"))
sys.path.insert(0, os.path.join(REPO, "oracle"))
import shard  # noqa: E402

OMEGAS = [0.05, 0.06, 0.07]


def _solve(omegas):
    import oracle_lib

    d = oracle_lib.load_deck(os.path.join(HERE, "golden", "config1", "input"))
    oc = oracle_lib.Case(d["xyz"], d["ncn"], d["ncon"], d["body_nelem"], d["xr"], d["h"], prepare=False)
    for k in ("xyz_p", "ds", "pnsz", "dxyz"):
        getattr(oc, k)[:] = d[k]
    oc.opts.nthread = 2
    betas = np.radians(d["wvhd"])
    return [oc.solve(oc.wave(om), betas)[:3] for om in omegas]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    lo, hi = shard.block(len(OMEGAS), rank, world)
    res = shard.gather_results(_solve(OMEGAS[lo:hi]), lo, dist, n=len(OMEGAS))
    slowest = shard.max_over_ranks(10.0 * (rank + 1), dist)
    if rank == 0:
        np.save(out, np.array([np.concatenate([np.ravel(a).view(np.float64) for a in r]) for r in res]))
        np.save(out + ".t.npy", np.array([slowest]))
    dist.barrier()
    dist.destroy_process_group()


def test_block_partition():
    for n in (1, 5, 40, 41):
        for world in (1, 2, 3, 8):
            spans = [shard.block(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [h - l for l, h in spans]
            assert max(sizes) - min(sizes) <= 1


@pytest.mark.timeout(600)
def test_two_gloo_ranks_match_single_process(tmp_path):
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = str(tmp_path / "res.npy")
    mp.start_processes(_rank, args=(2, port, out), nprocs=2, start_method="spawn", join=True)
    got = np.load(out)
    ref = np.array([np.concatenate([np.ravel(a).view(np.float64) for a in r]) for r in _solve(OMEGAS)])
    assert np.array_equal(got, ref)
    assert np.load(out + ".t.npy")[0] == 20.0
