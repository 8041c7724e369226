"""Heightfield edge cases on the device (needs a B200), against the
reference step by step (manifold.c:1924-2071, 1604-1616):

* a box wider than the window: the cell window clamps to 16 cells a side;
* a slab touching more than 64 triangles: the candidate lists fill and
  the triangle scan stops at the cap;
* a long capsule lying across many cells;
* bodies hanging over the grid's edge, and one beside the grid that
  never meets it (the window is empty: off the grid);
* a tilted, offset heightfield shape (local rotation and position on its
  static body), so the window is taken in the heightfield's own frame.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import cuda_available
from maul3d_b200 import abi

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


def _edge_world(lib, tilted: bool):
    wd = lib.m3DefaultWorldDef()
    wd.bodyCapacity = 32
    wd.shapeCapacity = 32
    wid = lib.m3CreateWorld(C.byref(wd))
    gd = lib.m3DefaultBodyDef()
    ground = lib.m3CreateBody(wid, C.byref(gd))
    sd = lib.m3DefaultShapeDef()
    plane = abi.m3Plane(abi.m3Vec3(0.0, 1.0, 0.0), -3.0)
    lib.m3CreatePlaneShape(ground, C.byref(sd), C.byref(plane))
    n = 40
    x = np.arange(n, dtype=np.float64)
    gx, gz = np.meshgrid(x, x)
    h = 0.35 * np.sin(0.4 * gx) * np.cos(0.3 * gz) + 0.1 * np.sin(1.3 * gx + 0.7 * gz)
    heights = (C.c_float * (n * n))(*[float(v) for v in h.astype(np.float32).ravel()])
    hd = lib.m3DefaultBodyDef()
    hd.position = abi.m3Pos3(-20.0, 0.0, -20.0)
    hbody = lib.m3CreateBody(wid, C.byref(hd))
    hsd = lib.m3DefaultShapeDef()
    if tilted:
        a = 0.06
        hsd.localRotation = abi.m3Quat(0.0, 0.0, float(np.sin(a / 2)), float(np.cos(a / 2)))
        hsd.localPosition = abi.m3Vec3(0.5, -0.2, 0.3)
    assert lib.m3CreateHeightFieldGridShape(hbody, C.byref(hsd), heights, n, n, 1.0).index1 > 0

    def body(x, y, z):
        bd = lib.m3DefaultBodyDef()
        bd.type = 2
        bd.position = abi.m3Pos3(x, y, z)
        return lib.m3CreateBody(wid, C.byref(bd))

    lib.m3CreateBoxShape(body(0.0, 1.6, 0.0), C.byref(sd), abi.m3Vec3(9.0, 0.5, 9.0))
    lib.m3CreateBoxShape(body(-10.0, 1.2, 10.0), C.byref(sd), abi.m3Vec3(4.0, 0.3, 4.0))
    cap = abi.m3Capsule(abi.m3Vec3(-7.0, 0.0, 0.0), abi.m3Vec3(7.0, 0.0, 0.0), 0.4)
    lib.m3CreateCapsuleShape(body(2.0, 1.4, -12.0), C.byref(sd), C.byref(cap))
    ball = abi.m3Sphere(abi.m3Vec3(0.0, 0.0, 0.0), 0.6)
    lib.m3CreateSphereShape(body(-20.2, 1.2, 5.0), C.byref(sd), C.byref(ball))
    lib.m3CreateBoxShape(body(19.0, 1.3, 19.2), C.byref(sd), abi.m3Vec3(0.6, 0.6, 0.6))
    lib.m3CreateSphereShape(body(30.0, 0.5, 0.0), C.byref(sd), C.byref(ball))
    for k in range(6):
        cap2 = abi.m3Capsule(abi.m3Vec3(0.0, -0.3, 0.0), abi.m3Vec3(0.0, 0.3, 0.0), 0.3)
        lib.m3CreateCapsuleShape(body(-15.0 + 5.0 * k, 1.5, 15.0), C.byref(sd), C.byref(cap2))
    return wid


@pytest.mark.parametrize("tilted", [False, True])
def test_heightfield_edge_cases_match_the_reference(m3, oracle, tilted):
    ours = abi.bind_create(m3.lib)
    ref = abi.bind_create(oracle.lib())
    g = m3.World(_edge_world(ours, tilted))
    r = oracle.RefWorld(_edge_world(ref, tilted))
    assert g.hash() == r.hash()
    for s in range(150):
        g.step(1.0 / 60.0, 4, 1)
        r.step(1.0 / 60.0, 4, 1)
        assert g.hash() == r.hash(), f"step {s + 1}"
