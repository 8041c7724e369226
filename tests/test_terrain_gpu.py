"""Heightfield terrain on the device (needs a B200).

Spheres, capsules and boxes dropped onto a seeded native heightfield
(shape.c:1175-1262) collide through the windowed triangle pipeline
(manifold.c:693-2071): the world hash must equal the reference's after
every step, snapshots after device steps must be the reference's bytes,
and a batch of terrain worlds (the per-family bucketed narrowphase, a
kernel of its own for heightfield pairs) must land where each world
stepped alone on the reference lands.  Integer and byte state compares
exactly.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import cuda_available
from maul3d_b200 import abi
from maul3d_b200.abi import SCENE_TERRAIN, SCENE_UNEVEN

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


def _snapshot(lib, wid) -> bytes:
    n = lib.m3World_SnapshotSize(wid)
    assert n > 0
    buf = (C.c_uint8 * n)()
    assert lib.m3World_Snapshot(wid, buf, n) == n
    return bytes(buf)


def _first_difference(a: bytes, b: bytes) -> str:
    if len(a) != len(b):
        return f"sizes {len(a)} vs {len(b)}"
    d = np.nonzero(np.frombuffer(a, np.uint8) != np.frombuffer(b, np.uint8))[0]
    return "equal" if len(d) == 0 else f"{len(d)} bytes differ, first at {int(d[0])}"


@pytest.fixture(scope="module")
def libs(m3, oracle):
    return abi.bind_snapshot(abi.bind_create(m3.lib)), abi.bind_snapshot(
        abi.bind_create(oracle.lib()))


@pytest.mark.parametrize("seed,bodies,steps", [(1, 12, 150), (2, 60, 120), (3, 150, 60)])
def test_terrain_every_step_matches_oracle(m3, oracle, seed, bodies, steps):
    g = m3.World.scene(SCENE_TERRAIN, seed, bodies)
    r = oracle.RefWorld.scene(SCENE_TERRAIN, seed, bodies)
    assert g.hash() == r.hash()
    for s in range(steps):
        g.step(1.0 / 60.0, 4, 1)
        r.step(1.0 / 60.0, 4, 1)
        assert g.hash() == r.hash(), f"seed {seed}: step {s + 1}"


def test_terrain_snapshot_after_device_steps(m3, oracle, libs):
    ours, ref = libs
    g = m3.World.scene(SCENE_TERRAIN, 7, 45)
    r = oracle.RefWorld.scene(SCENE_TERRAIN, 7, 45)
    done = 0
    for c in [1, 20, 80]:
        g.step(1.0 / 60.0, 4, c - done)
        r.step(1.0 / 60.0, 4, c - done)
        done = c
        a, b = _snapshot(ours, g.id), _snapshot(ref, r.id)
        assert a == b, f"step {c}: {_first_difference(a, b)}"


def test_restored_terrain_steps_like_the_reference(m3, oracle, libs):
    ours, ref = libs
    r = oracle.RefWorld.scene(SCENE_TERRAIN, 9, 80)
    r.step(1.0 / 60.0, 4, 30)
    snap = _snapshot(ref, r.id)
    g = m3.World.scene(SCENE_TERRAIN, 9, 80)
    g.step(1.0 / 60.0, 4, 2)  # device state the restore replaces
    buf = (C.c_uint8 * len(snap)).from_buffer_copy(snap)
    assert ours.m3World_Restore(g.id, buf, len(snap)), m3.last_error()
    for s in range(40):
        g.step(1.0 / 60.0, 4, 1)
        r.step(1.0 / 60.0, 4, 1)
        assert g.hash() == r.hash(), f"step {s + 1}"


def test_terrain_batch_equals_worlds_stepped_alone(m3, oracle):
    # Eight worlds, terrain and uneven mixed: more than the small-batch
    # bound, so pairs run bucketed by family.
    specs = [(SCENE_TERRAIN, 11 + k, 20 + 15 * k) for k in range(5)] + \
            [(SCENE_UNEVEN, 31 + k, 64 + 40 * k) for k in range(3)]
    batch = [m3.World.scene(*s) for s in specs]
    steps = 60
    m3.step_worlds(batch, 1.0 / 60.0, 4, steps)
    got = m3.hash_worlds(batch)
    for k, s in enumerate(specs):
        r = oracle.RefWorld.scene(*s)
        r.step(1.0 / 60.0, 4, steps)
        assert int(got[k]) == r.hash(), f"world {k} {s}"
