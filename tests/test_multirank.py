"""Root sharding across ranks (the N > 1 path), run as two gloo ranks on CPU.

Each rank plans its shard with the library's host-side planner, counts it with the CPU
oracle, and the counts are summed with one all_reduce, the same exchange bench.py does over
NCCL. The shards must partition the eligible roots and sum to the unsharded count."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.distributed as tdist
import torch.multiprocessing as mp

WORLD = 2


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank: int, port: int, result_dir: str):
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch

    import dumato_b200 as dm
    import oracle as orc
    from dumato_b200 import workloads

    tdist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=WORLD)
    g = workloads.make("er2k", 4)
    og = orc.OracleGraph.from_pairs(*g.edges())
    per = orc.clique_per_root(og, 4)
    roots, parts = dm.plan_roots(g, 4, True, dm.Options(rank=rank, world_size=WORLD))
    assert (parts == 0).all()
    mine = torch.tensor([int(per[roots].sum())], dtype=torch.int64)
    tdist.all_reduce(mine)
    gathered = [None] * WORLD
    tdist.all_gather_object(gathered, roots.tolist())
    d = dm.Dictionary.generate(4)
    q2c, _ = d.tables()
    mroots, _ = dm.plan_roots(g, 4, False, dm.Options(rank=rank, world_size=WORLD))
    h = torch.from_numpy(orc.motifs_roots(og, 4, q2c, d.n_classes, mroots).astype(np.int64))
    tdist.all_reduce(h)
    if rank == 0:
        all_roots = sorted(r for part in gathered for r in part)
        eligible = sorted(dm.plan_roots(g, 4, True)[0].tolist())
        np.save(os.path.join(result_dir, "res.npy"), np.array([
            int(mine.item()), orc.clique_dfs(og, 4), int(all_roots == eligible),
            int(len(set(gathered[0]) & set(gathered[1])) == 0),
            int(np.array_equal(h.numpy().astype(np.uint64), orc.motifs(og, 4, q2c, d.n_classes)))], dtype=np.int64))
    tdist.barrier()
    tdist.destroy_process_group()


def test_two_gloo_ranks_partition_and_sum(dm, orc, tmp_path):
    port = _free_port()
    mp.start_processes(_rank_main, args=(port, str(tmp_path)), nprocs=WORLD, start_method="spawn", join=True)
    sharded, total, cover, disjoint, motifs_ok = np.load(tmp_path / "res.npy").tolist()
    assert sharded == total and cover == 1 and disjoint == 1 and motifs_ok == 1
