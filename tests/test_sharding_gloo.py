"""The multi-rank path on CPU: a fixed list of worlds is split across two
gloo ranks by estimated cost (maul3d_b200.shard.partition), each rank
builds only its shard, steps it on its own (here on the host, through the
reference engine, since stepping on the device needs a GPU), and the
gathered per-world hashes equal those of the whole list stepped in one
process.  No data crosses ranks except the gathered hashes.
"""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from maul3d_b200.shard import partition, world_cost  # noqa: E402

SCENE_UNEVEN = 2
STEPS = 3
# (seed, dynamic bodies) of the fixed world list, deliberately uneven.
WORLDS = [(300 + i, n) for i, n in enumerate([32, 400, 48, 33, 260, 40, 96, 35, 180, 64])]


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
    from oracle import ref
    mine = partition([world_cost(n) for _, n in WORLDS], world_size)[rank]
    results = []
    for i in mine:
        seed, n = WORLDS[i]
        # The library builds the shard's world (creation bytes equal the
        # reference's), the reference engine steps it on this host.
        w = m3.World.scene(SCENE_UNEVEN, seed, n)
        r = ref.RefWorld.scene(SCENE_UNEVEN, seed, n)
        assert w.hash() == r.hash()
        r.step(1.0 / 60.0, 4, STEPS)
        results.append((i, r.hash()))
        r.destroy()
        w.destroy()
    gathered = [None] * world_size
    dist.all_gather_object(gathered, results)
    if rank == 0:
        import json
        Path(out_dir, "gathered.json").write_text(json.dumps(gathered))
    dist.barrier()
    dist.destroy_process_group()


def test_partition_balances_cost_and_covers_every_world_once():
    costs = [world_cost(n) for _, n in WORLDS]
    for ranks in (1, 2, 3, 4, 8):
        parts = partition(costs, ranks)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        # Longest-processing-time bound: no rank exceeds the mean by more
        # than the heaviest single world.
        assert max(loads) <= sum(costs) / ranks + max(costs)
        assert parts == partition(costs, ranks)  # deterministic
    assert world_cost(100, 7) == 107 and world_cost(100) == 400
    with pytest.raises(ValueError):
        partition(costs, 0)


def test_two_gloo_ranks_step_their_shards_without_exchange(tmp_path, oracle):
    port = _free_port()
    mp.spawn(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    import json
    gathered = json.loads((tmp_path / "gathered.json").read_text())
    assert len(gathered) == 2
    got = {i: h for shard in gathered for i, h in shard}
    assert sorted(got) == list(range(len(WORLDS))), "ranks dropped or duplicated worlds"
    assert all(len(shard) > 0 for shard in gathered)
    for i, (seed, n) in enumerate(WORLDS):
        r = oracle.RefWorld.scene(SCENE_UNEVEN, seed, n)
        r.step(1.0 / 60.0, 4, STEPS)
        assert r.hash() == got[i], f"world {i}"
        r.destroy()
