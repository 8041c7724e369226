"""Bullets in the continuous phase (needs a B200).

A bullet (m3BodyDef.isBullet) also sweeps against moving bodies, with the
target's own motion (solver.c:3237-3270).  Bullets fired down lanes at
free boxes, a box created between the bullets with one more bullet at
it, and a fast non-bullet sphere fired at a static block, in one world:
the world hash must equal the reference engine's after every step, and
the device must not refuse the world.
"""
import ctypes as C

import pytest

from conftest import cuda_available
from maul3d_b200 import abi

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

DT = 1.0 / 60.0


def _range_world(lib):
    wd = lib.m3DefaultWorldDef()
    wid = lib.m3CreateWorld(C.byref(wd))
    sd = lib.m3DefaultShapeDef()
    ground = lib.m3CreateBody(wid, C.byref(lib.m3DefaultBodyDef()))
    plane = abi.m3Plane(abi.m3Vec3(0.0, 1.0, 0.0), 0.0)
    lib.m3CreatePlaneShape(ground, C.byref(sd), C.byref(plane))
    # A static block in the last lane.
    bd = lib.m3DefaultBodyDef()
    bd.position = abi.m3Pos3(0.0, 0.5, 12.0)
    block = lib.m3CreateBody(wid, C.byref(bd))
    lib.m3CreateBoxShape(block, C.byref(sd), abi.m3Vec3(0.5, 0.5, 0.5))
    # Free boxes, one per lane, resting on the ground.
    for k, z in enumerate((-6.0, -3.0, 0.0, 3.0, 6.0)):
        bd = lib.m3DefaultBodyDef()
        bd.type = 2
        bd.position = abi.m3Pos3(0.5 * k, 0.5, z)
        box = lib.m3CreateBody(wid, C.byref(bd))
        lib.m3CreateBoxShape(box, C.byref(sd), abi.m3Vec3(0.5, 0.5, 0.5))
    # Bullets down the lanes at 60-100 m/s, created after the boxes (higher
    # body indices); then one more box and a bullet at it.
    speeds = (60.0, 75.0, 90.0, 100.0, 80.0)
    for k, z in enumerate((-6.0, -3.0, 0.0, 3.0, 6.0)):
        bd = lib.m3DefaultBodyDef()
        bd.type = 2
        bd.isBullet = True
        bd.position = abi.m3Pos3(-12.0, 0.5, z)
        bd.linearVelocity = abi.m3Vec3(speeds[k], 0.0, 0.0)
        ball = lib.m3CreateBody(wid, C.byref(bd))
        sphere = abi.m3Sphere(abi.m3Vec3(0.0, 0.0, 0.0), 0.1)
        lib.m3CreateSphereShape(ball, C.byref(sd), C.byref(sphere))
    bd = lib.m3DefaultBodyDef()
    bd.type = 2
    bd.position = abi.m3Pos3(3.0, 0.5, 9.0)
    late = lib.m3CreateBody(wid, C.byref(bd))
    lib.m3CreateBoxShape(late, C.byref(sd), abi.m3Vec3(0.4, 0.4, 0.4))
    bd = lib.m3DefaultBodyDef()
    bd.type = 2
    bd.isBullet = True
    bd.position = abi.m3Pos3(-12.0, 0.5, 9.0)
    bd.linearVelocity = abi.m3Vec3(70.0, 0.0, 0.0)
    ball = lib.m3CreateBody(wid, C.byref(bd))
    sphere = abi.m3Sphere(abi.m3Vec3(0.0, 0.0, 0.0), 0.1)
    lib.m3CreateSphereShape(ball, C.byref(sd), C.byref(sphere))
    # A fast non-bullet sphere at the static block.
    bd = lib.m3DefaultBodyDef()
    bd.type = 2
    bd.position = abi.m3Pos3(-12.0, 0.5, 12.0)
    bd.linearVelocity = abi.m3Vec3(80.0, 0.0, 0.0)
    ball = lib.m3CreateBody(wid, C.byref(bd))
    sphere = abi.m3Sphere(abi.m3Vec3(0.0, 0.0, 0.0), 0.1)
    lib.m3CreateSphereShape(ball, C.byref(sd), C.byref(sphere))
    return wid


def test_bullets_against_moving_targets_match_the_reference(m3, oracle):
    glib = abi.bind_create(m3.lib)
    rlib = abi.bind_create(oracle.lib())
    gid = _range_world(glib)
    rid = _range_world(rlib)
    g = m3.World(gid)
    assert g.hash() == rlib.m3World_Hash(rid)
    for s in range(60):
        glib.m3World_Step(gid, C.c_float(DT), 4)
        assert m3.last_error()[0] == 0, f"step {s + 1}: {m3.last_error()}"
        rlib.m3World_Step(rid, C.c_float(DT), 4)
        assert g.hash() == rlib.m3World_Hash(rid), f"step {s + 1}"
    glib.m3DestroyWorld(gid)
    rlib.m3DestroyWorld(rid)
