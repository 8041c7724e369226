"""Heightfield worlds on the host (no GPU): creation, its refusals and the
snapshot bytes against the reference (shape.c:1175-1262, broad_phase.c:
52-67 and 149-173, snapshot.c:274-279 and 568-594).

The tree leaf a heightfield enters with hangs from its body's origin with
a 0.1 margin, unlike every other shape's; the snapshot carries the
heightfield pool and each slot's samples after the hull content.  Both
are compared byte for byte with the reference's snapshot of the same
world, at creation and after a restore of a stepped reference world.
"""
import ctypes as C

import numpy as np
import pytest

from maul3d_b200 import abi
from maul3d_b200.abi import SCENE_SHOTS, SCENE_TERRAIN


@pytest.fixture(scope="module")
def libs(m3, oracle):
    return abi.bind_snapshot(abi.bind_create(m3.lib)), abi.bind_snapshot(
        abi.bind_create(oracle.lib()))


def _snapshot(lib, wid) -> bytes:
    n = lib.m3World_SnapshotSize(wid)
    assert n > 0
    buf = (C.c_uint8 * n)()
    assert lib.m3World_Snapshot(wid, buf, n) == n
    return bytes(buf)


@pytest.mark.parametrize("scene,seed,param", [(SCENE_TERRAIN, 1, 30), (SCENE_TERRAIN, 2, 200),
                                              (SCENE_TERRAIN, 3, 7), (SCENE_SHOTS, 3, 24),
                                              (SCENE_SHOTS, 4, 48)])
def test_terrain_world_at_creation_is_the_references(m3, oracle, libs, scene, seed, param):
    ours, ref = libs
    g = m3.World.scene(scene, seed, param)
    r = oracle.RefWorld.scene(scene, seed, param)
    assert g.hash() == r.hash()
    assert _snapshot(ours, g.id) == _snapshot(ref, r.id)


def test_restored_terrain_snapshot_round_trips(m3, oracle, libs):
    ours, ref = libs
    r = oracle.RefWorld.scene(SCENE_TERRAIN, 4, 60)
    r.step(1.0 / 60.0, 4, 25)
    snap = _snapshot(ref, r.id)
    g = m3.World.scene(SCENE_TERRAIN, 4, 60)
    buf = (C.c_uint8 * len(snap)).from_buffer_copy(snap)
    assert ours.m3World_Restore(g.id, buf, len(snap)), m3.last_error()
    assert g.hash() == r.hash()
    assert _snapshot(ours, g.id) == snap


def _try_grid(lib, wid, body_type, heights, nx, nz, cell):
    bd = lib.m3DefaultBodyDef()
    bd.type = body_type
    body = lib.m3CreateBody(wid, C.byref(bd))
    sd = lib.m3DefaultShapeDef()
    arr = (C.c_float * max(1, len(heights)))(*heights)
    return lib.m3CreateHeightFieldGridShape(body, C.byref(sd), arr, nx, nz, cell).index1 > 0


@pytest.mark.parametrize("case", ["ok", "one_row", "too_wide", "zero_cell", "nan_sample",
                                  "dynamic_body"])
def test_heightfield_creation_refusals_match(m3, oracle, libs, case):
    ours, ref = libs
    nx, nz, cell, body_type = 4, 3, 1.0, 0
    heights = [0.1 * k for k in range(nx * nz)]
    if case == "one_row":
        nz = 1
        heights = heights[:nx]
    elif case == "too_wide":
        nx, nz = 256, 2
        heights = [0.0] * (nx * nz)
    elif case == "zero_cell":
        cell = 0.0
    elif case == "nan_sample":
        heights[5] = float("nan")
    elif case == "dynamic_body":
        body_type = 2
    results = []
    for lib in (ours, ref):
        wd = lib.m3DefaultWorldDef()
        wid = lib.m3CreateWorld(C.byref(wd))
        results.append(_try_grid(lib, wid, body_type, heights, nx, nz, cell))
        lib.m3DestroyWorld(wid)
    assert results[0] == results[1] == (case == "ok")
