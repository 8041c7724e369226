"""General convex hulls on the device (needs a B200).

The reference builds worlds of QuickHull hulls from seeded point clouds
(16-32 points in the unit ball, scaled 0.5-1.5: the rain configuration's
hulls, shape.h:143-149), mixed with spheres and capsules on a plane; the
snapshot restores into this library and both engines step it, the world
hashes compared after every step.  This drives the hull paths of the
narrowphase (hull-hull SAT and clipping with many faces and edges,
plane-hull, GJK against round shapes, capsule-hull) and the contact
solver with general manifolds.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import cuda_available
from maul3d_b200 import abi

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


def _hull_world(lib, seed: int, bodies: int):
    rng = np.random.default_rng(seed)
    wd = lib.m3DefaultWorldDef()
    wd.bodyCapacity = bodies + 4
    wd.shapeCapacity = bodies + 4
    wid = lib.m3CreateWorld(C.byref(wd))
    gd = lib.m3DefaultBodyDef()
    ground = lib.m3CreateBody(wid, C.byref(gd))
    sd = lib.m3DefaultShapeDef()
    plane = abi.m3Plane(abi.m3Vec3(0.0, 1.0, 0.0), 0.0)
    lib.m3CreatePlaneShape(ground, C.byref(sd), C.byref(plane))
    # Layers of a 4 x 4 column grid, 3.2 m apart, jittered: the bodies
    # land on the plane and on each other.
    made = 0
    for k in range(bodies):
        bd = lib.m3DefaultBodyDef()
        bd.type = 2
        layer, cell = divmod(k, 16)
        bd.position = abi.m3Pos3(3.2 * (cell % 4) + rng.uniform(-0.6, 0.6),
                                 1.6 + 3.2 * layer + rng.uniform(0, 0.5),
                                 3.2 * (cell // 4) + rng.uniform(-0.6, 0.6))
        bd.angularVelocity = abi.m3Vec3(*[float(x) for x in rng.uniform(-1, 1, 3)])
        body = lib.m3CreateBody(wid, C.byref(bd))
        sd = lib.m3DefaultShapeDef()
        sd.density = float(rng.uniform(0.5, 2.0))
        sd.friction = float(rng.uniform(0.3, 0.9))
        kind = k % 5
        if kind < 3:
            n = int(rng.integers(16, 33))
            pts = rng.normal(size=(n, 3))
            pts *= (rng.uniform(0, 1, (n, 1)) ** (1 / 3)) / np.linalg.norm(pts, axis=1, keepdims=True)
            pts *= rng.uniform(0.5, 1.5)
            arr = (abi.m3Vec3 * n)(*[abi.m3Vec3(*[float(c) for c in p]) for p in pts.astype(np.float32)])
            sid = lib.m3CreateHullShape(body, C.byref(sd), arr, n)
            made += sid.index1 > 0
        elif kind == 3:
            ball = abi.m3Sphere(abi.m3Vec3(0.0, 0.0, 0.0), float(rng.uniform(0.25, 0.75)))
            lib.m3CreateSphereShape(body, C.byref(sd), C.byref(ball))
        else:
            hh = float(rng.uniform(0.3, 1.0))
            cap = abi.m3Capsule(abi.m3Vec3(0.0, -hh, 0.0), abi.m3Vec3(0.0, hh, 0.0),
                                float(rng.uniform(0.2, 0.5)))
            lib.m3CreateCapsuleShape(body, C.byref(sd), C.byref(cap))
    assert made > 0
    return wid, wd


@pytest.mark.parametrize("seed,bodies,steps", [(1, 40, 200), (2, 150, 150)])
def test_quickhull_worlds_step_like_the_reference(m3, oracle, seed, bodies, steps):
    ref = abi.bind_snapshot(abi.bind_create(oracle.lib()))
    ref.m3CreateHullShape.argtypes = [abi.m3BodyId, C.POINTER(abi.m3ShapeDef),
                                      C.POINTER(abi.m3Vec3), C.c_int32]
    ref.m3CreateHullShape.restype = abi.m3ShapeId
    ours = abi.bind_snapshot(abi.bind_create(m3.lib))
    rid, wd = _hull_world(ref, seed, bodies)
    r = oracle.RefWorld(rid)
    n = ref.m3World_SnapshotSize(rid)
    snap = (C.c_uint8 * n)()
    assert ref.m3World_Snapshot(rid, snap, n) == n
    gid = ours.m3CreateWorld(C.byref(wd))
    assert ours.m3World_Restore(gid, snap, n), m3.last_error()
    g = m3.World(gid)
    assert g.hash() == r.hash()
    for s in range(steps):
        r.step(1.0 / 60.0, 4, 1)
        g.step(1.0 / 60.0, 4, 1)
        if g.hash() != r.hash():
            pytest.fail(f"step {s + 1}: {g.state().first_difference(r.state())}")


def _rain_world(lib, seed: int, bodies: int):
    """A reduced rain field (the mixed rain configuration's shapes): 40 %
    spheres, 30 % capsules and 30 % QuickHull hulls from 16-32 points,
    dropped from 5-30 m onto a heightfield of four seeded sine octaves
    (4 m amplitude, 1 m cells), density U[0.5, 2], friction U[0.3, 0.9]."""
    rng = np.random.default_rng(seed)
    n = 72
    wd = lib.m3DefaultWorldDef()
    wd.bodyCapacity = bodies + 4
    wd.shapeCapacity = bodies + 4
    wid = lib.m3CreateWorld(C.byref(wd))
    x = np.arange(n, dtype=np.float64)
    gx, gz = np.meshgrid(x, x)
    h = np.zeros_like(gx)
    for octave in range(4):
        f = 0.05 * 2 ** octave
        ph = rng.uniform(0, 2 * np.pi, 2)
        h += (4.0 / 2 ** octave) * np.sin(f * gx + ph[0]) * np.cos(f * gz + ph[1]) / 1.875
    heights = (C.c_float * (n * n))(*[float(v) for v in h.astype(np.float32).ravel()])
    gd = lib.m3DefaultBodyDef()
    gd.position = abi.m3Pos3(-0.5 * (n - 1), 0.0, -0.5 * (n - 1))
    ground = lib.m3CreateBody(wid, C.byref(gd))
    sd = lib.m3DefaultShapeDef()
    hf = lib.m3CreateHeightFieldGridShape(ground, C.byref(sd), heights, n, n, 1.0)
    assert hf.index1 > 0
    side = int(np.ceil(np.sqrt(bodies)))
    spacing = (n - 12) / side
    for k in range(bodies):
        bd = lib.m3DefaultBodyDef()
        bd.type = 2
        bd.position = abi.m3Pos3(-0.5 * (n - 12) + spacing * (k % side) + rng.uniform(-0.3, 0.3),
                                 float(rng.uniform(5.0, 30.0)),
                                 -0.5 * (n - 12) + spacing * (k // side) + rng.uniform(-0.3, 0.3))
        body = lib.m3CreateBody(wid, C.byref(bd))
        sd = lib.m3DefaultShapeDef()
        sd.density = float(rng.uniform(0.5, 2.0))
        sd.friction = float(rng.uniform(0.3, 0.9))
        u = k % 10
        if u < 4:
            ball = abi.m3Sphere(abi.m3Vec3(0.0, 0.0, 0.0), float(rng.uniform(0.25, 0.75)))
            lib.m3CreateSphereShape(body, C.byref(sd), C.byref(ball))
        elif u < 7:
            hh = float(rng.uniform(0.3, 1.0))
            cap = abi.m3Capsule(abi.m3Vec3(0.0, -hh, 0.0), abi.m3Vec3(0.0, hh, 0.0),
                                float(rng.uniform(0.2, 0.5)))
            lib.m3CreateCapsuleShape(body, C.byref(sd), C.byref(cap))
        else:
            m = int(rng.integers(16, 33))
            pts = rng.normal(size=(m, 3))
            pts *= (rng.uniform(0, 1, (m, 1)) ** (1 / 3)) / np.linalg.norm(pts, axis=1, keepdims=True)
            pts *= rng.uniform(0.5, 1.5)
            arr = (abi.m3Vec3 * m)(*[abi.m3Vec3(*[float(c) for c in p]) for p in pts.astype(np.float32)])
            lib.m3CreateHullShape(body, C.byref(sd), arr, m)
    return wid, wd


@pytest.mark.parametrize("seed,bodies,steps", [(3, 120, 180)])
def test_rain_field_on_terrain_steps_like_the_reference(m3, oracle, seed, bodies, steps):
    # Fast falls over the heightfield run the continuous phase, hulls meet
    # the heightfield through the hull-triangle kernel.
    ref = abi.bind_snapshot(abi.bind_create(oracle.lib()))
    ref.m3CreateHullShape.argtypes = [abi.m3BodyId, C.POINTER(abi.m3ShapeDef),
                                      C.POINTER(abi.m3Vec3), C.c_int32]
    ref.m3CreateHullShape.restype = abi.m3ShapeId
    ref.m3CreateHeightFieldGridShape.argtypes = [abi.m3BodyId, C.POINTER(abi.m3ShapeDef),
                                                 C.POINTER(C.c_float), C.c_int32, C.c_int32,
                                                 C.c_float]
    ref.m3CreateHeightFieldGridShape.restype = abi.m3ShapeId
    ours = abi.bind_snapshot(abi.bind_create(m3.lib))
    rid, wd = _rain_world(ref, seed, bodies)
    r = oracle.RefWorld(rid)
    n = ref.m3World_SnapshotSize(rid)
    snap = (C.c_uint8 * n)()
    assert ref.m3World_Snapshot(rid, snap, n) == n
    gid = ours.m3CreateWorld(C.byref(wd))
    assert ours.m3World_Restore(gid, snap, n), m3.last_error()
    g = m3.World(gid)
    assert g.hash() == r.hash()
    for s in range(steps):
        r.step(1.0 / 60.0, 4, 1)
        g.step(1.0 / 60.0, 4, 1)
        if g.hash() != r.hash():
            pytest.fail(f"step {s + 1}: {g.state().first_difference(r.state())}")
