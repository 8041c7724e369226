"""Snapshots of worlds stepped on the GPU, and journals replayed there
(needs a B200).

A snapshot after device steps must be the reference's bytes after the
same steps: the broadphase tree the device refreshes every step
(broad_phase.c:500-539), the pair arrays past the live list, the pools.
A world restored from a reference snapshot and stepped on the device, or
driven by a journal of impulses and steps, must land on the reference's
hash and bytes (snapshot.c:680-931, world.c:1505-3218).
"""
import ctypes as C

import numpy as np
import pytest

from conftest import cuda_available
from maul3d_b200 import abi
from maul3d_b200.abi import SCENE_BOX_PYRAMID, SCENE_TOWERS, SCENE_UNEVEN

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


def _snapshot(lib, wid) -> bytes:
    n = lib.m3World_SnapshotSize(wid)
    assert n > 0
    buf = (C.c_uint8 * n)()
    assert lib.m3World_Snapshot(wid, buf, n) == n
    return bytes(buf)


def _restore(lib, wid, data: bytes) -> bool:
    buf = (C.c_uint8 * len(data)).from_buffer_copy(data)
    return bool(lib.m3World_Restore(wid, buf, len(data)))


def _replay(lib, wid, data: bytes) -> bool:
    buf = (C.c_uint8 * max(len(data), 1)).from_buffer_copy(data or b"\0")
    return bool(lib.m3World_JournalReplay(wid, buf, len(data)))


def _first_difference(a: bytes, b: bytes) -> str:
    if len(a) != len(b):
        return f"sizes {len(a)} vs {len(b)}"
    x = np.frombuffer(a, np.uint8)
    y = np.frombuffer(b, np.uint8)
    d = np.nonzero(x != y)[0]
    return "equal" if len(d) == 0 else f"{len(d)} bytes differ, first at {int(d[0])}"


@pytest.fixture(scope="module")
def libs(m3, oracle):
    ref = abi.bind_snapshot(abi.bind_create(oracle.lib()))
    ours = abi.bind_snapshot(abi.bind_create(m3.lib))
    return ours, ref


@pytest.mark.parametrize("scene,seed,param,checkpoints", [
    (SCENE_BOX_PYRAMID, 0, 20, [1, 30, 120]),
    (SCENE_UNEVEN, 11, 48, [1, 10, 60, 150]),
    (SCENE_UNEVEN, 12, 300, [5, 50]),
    (SCENE_TOWERS, 7, 4, [1, 20, 90]),
])
def test_snapshot_after_device_steps_is_the_references(m3, oracle, libs, scene, seed, param,
                                                        checkpoints):
    ours, ref = libs
    g = m3.World.scene(scene, seed, param)
    r = oracle.RefWorld.scene(scene, seed, param)
    done = 0
    for c in checkpoints:
        g.step(1.0 / 60.0, 4, c - done)
        r.step(1.0 / 60.0, 4, c - done)
        done = c
        a, b = _snapshot(ours, g.id), _snapshot(ref, r.id)
        assert a == b, f"step {c}: {_first_difference(a, b)}"


def test_restored_world_steps_on_the_device_like_the_reference(m3, oracle, libs):
    ours, ref = libs
    r = oracle.RefWorld.scene(SCENE_UNEVEN, 31, 200)
    r.step(1.0 / 60.0, 4, 40)
    snap = _snapshot(ref, r.id)
    g = m3.World.scene(SCENE_UNEVEN, 31, 200)
    g.step(1.0 / 60.0, 4, 3)  # device-resident state the restore replaces
    assert _restore(ours, g.id, snap)
    for s in range(30):
        g.step(1.0 / 60.0, 4, 1)
        r.step(1.0 / 60.0, 4, 1)
        assert g.hash() == r.hash(), f"step {s + 1}"
    a, b = _snapshot(ours, g.id), _snapshot(ref, r.id)
    assert a == b, _first_difference(a, b)


def test_journal_of_impulses_and_steps_replays_like_the_reference(m3, oracle, libs):
    # The serving request shape: a snapshot plus frames of linear
    # impulses on a few bodies, each closed by a step.
    ours, ref = libs
    r = oracle.RefWorld.scene(SCENE_UNEVEN, 41, 240)
    r.step(1.0 / 60.0, 4, 30)
    snap = _snapshot(ref, r.id)
    g = m3.World.scene(SCENE_UNEVEN, 41, 240)
    assert _restore(ours, g.id, snap)
    rng = np.random.default_rng(41)
    journal = b""
    for frame in range(12):
        for _ in range(int(rng.integers(1, 9))):
            body = int(rng.integers(2, 200))
            mag = float(rng.uniform(1.0, 50.0))
            d = rng.normal(size=3)
            d = (d / np.linalg.norm(d) * mag).astype(np.float32)
            journal += abi.journal_body_command(abi.OP_APPLY_LINEAR_IMPULSE, body, 0,
                                               [float(x) for x in d])
        journal += abi.journal_step(1.0 / 60.0, 4)
    assert _replay(ref, r.id, journal)
    assert _replay(ours, g.id, journal), m3.last_error()
    assert g.hash() == r.hash()
    a, b = _snapshot(ours, g.id), _snapshot(ref, r.id)
    assert a == b, _first_difference(a, b)
