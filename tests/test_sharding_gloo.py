"""The multi-rank path on CPU: two gloo ranks each build their shard of
the batched workload (no exchange on the data path), and the gathered
per-world hashes equal the reference's for every world of both shards.
(Stepping needs a GPU; the shards' creation-time hashes are computed on
the host, the same hash the device reproduces after every step.)
"""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world_size: int, port: int, out_dir: str) -> None:
    sys.path.insert(0, str(ROOT))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world_size,
                            timeout=timedelta(seconds=60))
    import maul3d_b200 as m3
    from maul3d_b200.shard import rank_seed, shard_sizes
    seed = rank_seed(7, rank)
    sizes = shard_sizes(m3.lib, seed, 6, 32, 256)
    hashes = []
    for i, n in enumerate(sizes):
        w = m3.World.scene(2, seed + i, n)
        hashes.append((seed + i, n, w.hash()))
        w.destroy()
    gathered = [None] * world_size
    dist.all_gather_object(gathered, hashes)
    if rank == 0:
        import json
        Path(out_dir, "gathered.json").write_text(json.dumps(gathered))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_shard_worlds_without_exchange(tmp_path, oracle):
    port = _free_port()
    mp.spawn(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    import json
    gathered = json.loads((tmp_path / "gathered.json").read_text())
    assert len(gathered) == 2
    seeds = [s for shard in gathered for s, _, _ in shard]
    assert len(set(seeds)) == len(seeds), "ranks built overlapping worlds"
    for shard in gathered:
        for seed, n, h in shard:
            r = oracle.RefWorld.scene(2, seed, n)
            assert r.hash() == h
            r.destroy()
