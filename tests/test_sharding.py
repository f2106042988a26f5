"""Instances over ranks (mit_jax_b200/sharding.py) on two CPU processes with the gloo backend: the shards are
disjoint, cover the batch and balance the work; each rank solves its shard (oracle, small LLC grid); the gathered
diagnostics equal a one-process solve of the whole batch; the job time is the max over ranks."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from mit_jax_b200.sharding import estimated_work, shard_instances


def test_shards_disjoint_cover_and_balance():
    work = estimated_work([105300] * 7 + [947700] * 3, [230, 240, 250, 235, 245, 231, 239, 300, 280, 290])
    for world in (1, 2, 3, 4):
        parts = [shard_instances(work, world, r) for r in range(world)]
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(work)))
        loads = [work[p].sum() for p in parts]
        assert max(loads) - min(loads) <= work.max()
    with pytest.raises(ValueError):
        shard_instances(work, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    import torch.distributed as dist
    from mit_jax_b200.sharding import gather_records, max_over_ranks
    from mit_jax_b200.synthetic import make_batch
    from oracle import cg2d_oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n = 5
        mine = shard_instances(estimated_work([1] * n), world, rank)
        syn, B = make_batch(16, ts=8, members=mine)
        recs = []
        for k, m in enumerate(mine):
            ops = tuple(B[name][k] for name in ("aW2d", "aS2d", "aC2d", "pW", "pS", "pC"))
            x, d = O.cg2d_fortran(syn.L, syn.topo.maps["T"], ops, B["b"][k], B["x0"][k], cg2dNorm=B["cg2dNorm"][k],
                                  tolerance=1e-10, max_iters=200, sum_order="rowblock")
            recs.append((m, int(d["numIters"]), float(np.abs(x).sum())))
        everything = gather_records(recs)
        slowest = max_over_ranks(10.0 + rank)
        if rank == 0:
            np.save(os.path.join(out_dir, "gathered.npy"), np.asarray(everything, dtype=np.float64))
            np.save(os.path.join(out_dir, "slowest.npy"), np.asarray([slowest]))
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo(tmp_path):
    world, port = 2, _free_port()
    mp.start_processes(_rank, args=(world, port, str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    got = np.load(tmp_path / "gathered.npy")
    assert float(np.load(tmp_path / "slowest.npy")[0]) == 11.0
    assert sorted(got[:, 0].astype(int).tolist()) == list(range(5))
    # the same instances solved in this process, one after another
    from mit_jax_b200.synthetic import make_batch
    from oracle import cg2d_oracle as O
    syn, B = make_batch(16, ts=8, members=list(range(5)))
    for m, iters, csum in got:
        m = int(m)
        ops = tuple(B[name][m] for name in ("aW2d", "aS2d", "aC2d", "pW", "pS", "pC"))
        x, d = O.cg2d_fortran(syn.L, syn.topo.maps["T"], ops, B["b"][m], B["x0"][m], cg2dNorm=B["cg2dNorm"][m],
                              tolerance=1e-10, max_iters=200, sum_order="rowblock")
        assert int(d["numIters"]) == int(iters)
        assert float(np.abs(x).sum()) == csum
