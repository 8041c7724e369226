"""Hull shapes from point clouds (CPU): m3CreateHullShape builds the same
hull slab as the reference's QuickHull (shape.c:988-1030,
quickhull.c:1110-1216) for every cloud, and refuses the same clouds.

Each case builds a world holding one body per cloud in both engines;
the world hashes and the snapshot bytes (which carry every interned hull
slab byte for byte, snapshot.c) must be equal, and a refused cloud must
be refused by both.  Clouds: uniform in a ball (the rain and serving
configurations' hulls, 16-32 and 16 points), on a sphere, box corners
with jitter, duplicates, near-coplanar and collinear sets, large
coordinates far from the origin, and the 4- and 256-point limits.
"""
import ctypes as C

import numpy as np
import pytest

from maul3d_b200 import abi


def _clouds(seed: int):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(12):
        n = int(rng.integers(16, 33))
        p = rng.normal(size=(n, 3))
        p *= (rng.uniform(0, 1, (n, 1)) ** (1 / 3)) / np.linalg.norm(p, axis=1, keepdims=True)
        out.append(p * rng.uniform(0.5, 1.5))
    for n in (16, 64, 200):
        p = rng.normal(size=(n, 3))
        out.append(p / np.linalg.norm(p, axis=1, keepdims=True) * 0.8)
    corners = np.array([[x, y, z] for x in (-1, 1) for y in (-1, 1) for z in (-1, 1)], float)
    out.append(corners * 0.5)
    out.append(corners * 0.5 + rng.normal(scale=1e-4, size=corners.shape))
    out.append(np.concatenate([corners, corners, corners[:3]]) * 0.7)
    flat = rng.uniform(-1, 1, (20, 3))
    flat[:, 1] = rng.normal(scale=1e-7, size=20)
    out.append(flat)
    line = np.outer(rng.uniform(-1, 1, 12), [1.0, 2.0, 0.5])
    out.append(line)
    out.append(rng.uniform(-1, 1, (24, 3)) + np.array([5000.0, -3000.0, 250.0]))
    out.append(rng.uniform(-1, 1, (4, 3)))
    out.append(rng.uniform(-2, 2, (256, 3)))
    out.append(rng.uniform(-1, 1, (3, 3)))
    out.append(rng.uniform(-1, 1, (257, 3)))
    return [c.astype(np.float32) for c in out]


def _build(lib, clouds):
    wd = lib.m3DefaultWorldDef()
    wd.bodyCapacity = len(clouds) + 4
    wd.shapeCapacity = len(clouds) + 4
    wid = lib.m3CreateWorld(C.byref(wd))
    made = []
    for k, cloud in enumerate(clouds):
        bd = lib.m3DefaultBodyDef()
        bd.type = 2
        bd.position = abi.m3Pos3(3.0 * k, 1.0, 0.0)
        body = lib.m3CreateBody(wid, C.byref(bd))
        sd = lib.m3DefaultShapeDef()
        sd.density = 1.0 + 0.1 * k
        arr = (abi.m3Vec3 * len(cloud))(*[abi.m3Vec3(*[float(c) for c in p]) for p in cloud])
        sid = lib.m3CreateHullShape(body, C.byref(sd), arr, len(cloud))
        made.append(sid.index1 > 0)
    return wid, made


@pytest.mark.parametrize("seed", [1, 2, 3, 4])
def test_hull_slabs_and_refusals_match_the_reference(m3, oracle, seed):
    ours = abi.bind_snapshot(abi.bind_create(m3.lib))
    ref = abi.bind_snapshot(abi.bind_create(oracle.lib()))
    clouds = _clouds(seed)
    gid, gmade = _build(ours, clouds)
    rid, rmade = _build(ref, clouds)
    assert gmade == rmade
    assert sum(gmade) >= len(clouds) - 5  # the degenerate few are refused
    assert ours.m3World_Hash(gid) == ref.m3World_Hash(rid)
    n = ref.m3World_SnapshotSize(rid)
    assert ours.m3World_SnapshotSize(gid) == n
    a = (C.c_uint8 * n)()
    b = (C.c_uint8 * n)()
    assert ref.m3World_Snapshot(rid, a, n) == n
    assert ours.m3World_Snapshot(gid, b, n) == n
    assert bytes(a) == bytes(b)
    ours.m3DestroyWorld(gid)
    ref.m3DestroyWorld(rid)


def test_hull_refusals(m3):
    lib = abi.bind_create(m3.lib)
    wid = lib.m3CreateWorld(C.byref(lib.m3DefaultWorldDef()))
    bd = lib.m3DefaultBodyDef()
    bd.type = 2
    body = lib.m3CreateBody(wid, C.byref(bd))
    sd = lib.m3DefaultShapeDef()
    pts = (abi.m3Vec3 * 4)(abi.m3Vec3(0, 0, 0), abi.m3Vec3(1, 0, 0), abi.m3Vec3(0, 1, 0),
                           abi.m3Vec3(0, 0, float("nan")))
    assert lib.m3CreateHullShape(body, C.byref(sd), pts, 4).index1 == 0
    assert m3.last_error()[0] == m3.M3GPU_ERR_INVALID
    assert lib.m3CreateHullShape(body, C.byref(sd), None, 4).index1 == 0
    assert lib.m3CreateHullShape(body, C.byref(sd), pts, 0).index1 == 0
    lib.m3DestroyWorld(wid)
