"""Event streams of the last step (needs a B200).

Contact begin/end, sensor begin/end, joint-break, body move and hit
events (world.h:207-313) must be the reference's, stream for stream and
in the same order, after every step: bodies settling and bouncing
(contacts begin and end, bodies falling asleep), towers whose welds break
(joint-break events with the ids the joints had), spheres falling
through a sensor box (sensor streams), and bodies landing on a ground
that asks for hit events.  Body move and hit events carry transforms,
points, normals and speeds, compared byte for byte.  A restore clears
every stream in both engines.
"""
import collections
import ctypes as C

import pytest

from conftest import cuda_available
from maul3d_b200 import abi
from maul3d_b200.abi import SCENE_BOUNCE, SCENE_CITY, SCENE_TOWERS, SCENE_UNEVEN

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

DT = 1.0 / 60.0


@pytest.fixture(scope="module")
def libs(m3, oracle):
    return abi.bind_events(m3.lib), abi.bind_events(oracle.lib())


def _compare(glib, rlib, gid, rid, where):
    got = abi.read_events(glib, gid)
    want = abi.read_events(rlib, rid)
    for name in want:
        assert got[name] == want[name], f"{where}: {name}"
    return want


@pytest.mark.parametrize("scene,seed,param,substeps,steps", [
    (SCENE_UNEVEN, 71, 300, 4, 90),
    (SCENE_BOUNCE, 72, 60, 4, 120),
    (SCENE_TOWERS, 73, 6, 4, 90),
    (SCENE_CITY, 74, 3, 8, 45),
])
def test_event_streams_equal_the_reference_every_step(m3, oracle, libs, scene, seed, param,
                                                      substeps, steps):
    glib, rlib = libs
    g = m3.World.scene(scene, seed, param)
    r = oracle.RefWorld.scene(scene, seed, param)
    seen = collections.Counter()
    for s in range(steps):
        g.step(DT, substeps, 1)
        r.step(DT, substeps, 1)
        want = _compare(glib, rlib, g.id, r.id, f"step {s + 1}")
        for name, events in want.items():
            if isinstance(events, list):
                seen[name] += len(events)
    assert g.hash() == r.hash()
    # The scenes do what they are here for.
    assert seen["m3World_ContactBeginEvents"] > 0
    assert seen["m3World_BodyMoveEvents"] > 0
    if scene in (SCENE_UNEVEN, SCENE_BOUNCE):
        assert seen["m3World_ContactEndEvents"] > 0
    if scene == SCENE_CITY:
        assert seen["m3World_JointBreakEvents"] > 0
    g.destroy()
    r.destroy()


def _sensor_world(lib):
    """A ground plane, a static sensor box (4 x 1 x 4 at height 3) and
    spheres dropped through it from different heights."""
    wd = lib.m3DefaultWorldDef()
    wid = lib.m3CreateWorld(C.byref(wd))
    sd = lib.m3DefaultShapeDef()
    ground = lib.m3CreateBody(wid, C.byref(lib.m3DefaultBodyDef()))
    plane = abi.m3Plane(abi.m3Vec3(0.0, 1.0, 0.0), 0.0)
    lib.m3CreatePlaneShape(ground, C.byref(sd), C.byref(plane))
    bd = lib.m3DefaultBodyDef()
    bd.position = abi.m3Pos3(0.0, 3.0, 0.0)
    gate = lib.m3CreateBody(wid, C.byref(bd))
    sensor = lib.m3DefaultShapeDef()
    sensor.isSensor = True
    lib.m3CreateBoxShape(gate, C.byref(sensor), abi.m3Vec3(2.0, 0.5, 2.0))
    for k in range(6):
        bd = lib.m3DefaultBodyDef()
        bd.type = 2
        bd.position = abi.m3Pos3(-1.5 + 0.6 * k, 5.0 + 0.7 * k, 0.3 * (k % 3) - 0.3)
        body = lib.m3CreateBody(wid, C.byref(bd))
        sphere = abi.m3Sphere(abi.m3Vec3(0.0, 0.0, 0.0), 0.25)
        lib.m3CreateSphereShape(body, C.byref(sd), C.byref(sphere))
    return wid


def test_sensor_streams_equal_the_reference(m3, oracle, libs):
    glib, rlib = libs
    gc = abi.bind_create(glib)
    rc = abi.bind_create(rlib)
    gid = _sensor_world(gc)
    rid = _sensor_world(rc)
    g = m3.World(gid)
    seen_begin = 0
    seen_end = 0
    for s in range(150):
        glib.m3World_Step(gid, C.c_float(DT), 4)
        rlib.m3World_Step(rid, C.c_float(DT), 4)
        want = _compare(glib, rlib, gid, rid, f"step {s + 1}")
        seen_begin += len(want["m3World_SensorBeginEvents"])
        seen_end += len(want["m3World_SensorEndEvents"])
    assert seen_begin == 6 and seen_end == 6
    assert g.hash() == rlib.m3World_Hash(rid)
    glib.m3DestroyWorld(gid)
    rlib.m3DestroyWorld(rid)


def _restore(lib, wid, data: bytes) -> bool:
    buf = (C.c_uint8 * len(data)).from_buffer_copy(data)
    return bool(lib.m3World_Restore(wid, buf, len(data)))


def test_restore_clears_the_streams(m3, oracle, libs):
    glib, rlib = libs
    abi.bind_snapshot(glib)
    abi.bind_snapshot(rlib)
    g = m3.World.scene(SCENE_BOUNCE, 75, 40)
    r = oracle.RefWorld.scene(SCENE_BOUNCE, 75, 40)
    for _ in range(30):
        g.step(DT, 4, 1)
        r.step(DT, 4, 1)
    snap = m3.snapshot(g)
    g.step(DT, 4, 1)
    r.step(DT, 4, 1)
    _compare(glib, rlib, g.id, r.id, "before the restore")
    assert _restore(glib, g.id, snap)
    assert _restore(rlib, r.id, snap)
    after = _compare(glib, rlib, g.id, r.id, "after the restore")
    assert all((len(v) if isinstance(v, list) else v) == 0 for v in after.values())
    # The next step's streams again equal the reference's.
    g.step(DT, 4, 1)
    r.step(DT, 4, 1)
    _compare(glib, rlib, g.id, r.id, "first step after the restore")
    assert g.hash() == r.hash()
    g.destroy()
    r.destroy()


def _hit_world(lib):
    """A ground plane with hit events enabled; spheres and boxes dropped
    from 1-6 m, some thrown sideways, one box with hit events of its own
    landing on a sphere-free patch."""
    wd = lib.m3DefaultWorldDef()
    wid = lib.m3CreateWorld(C.byref(wd))
    ground = lib.m3CreateBody(wid, C.byref(lib.m3DefaultBodyDef()))
    gsd = lib.m3DefaultShapeDef()
    gsd.enableHitEvents = True
    plane = abi.m3Plane(abi.m3Vec3(0.0, 1.0, 0.0), 0.0)
    lib.m3CreatePlaneShape(ground, C.byref(gsd), C.byref(plane))
    sd = lib.m3DefaultShapeDef()
    sd.restitution = 0.4
    for k in range(12):
        bd = lib.m3DefaultBodyDef()
        bd.type = 2
        bd.position = abi.m3Pos3(-6.0 + 1.1 * k, 1.0 + 0.45 * k, 0.5 * (k % 3))
        bd.linearVelocity = abi.m3Vec3(1.5 * ((k % 4) - 1.5), 0.0, 0.0)
        body = lib.m3CreateBody(wid, C.byref(bd))
        if k % 2 == 0:
            sphere = abi.m3Sphere(abi.m3Vec3(0.0, 0.0, 0.0), 0.3)
            lib.m3CreateSphereShape(body, C.byref(sd), C.byref(sphere))
        else:
            own = lib.m3DefaultShapeDef()
            own.enableHitEvents = k == 5
            lib.m3CreateBoxShape(body, C.byref(own), abi.m3Vec3(0.3, 0.25, 0.35))
    return wid


def test_hit_events_equal_the_reference(m3, oracle, libs):
    glib, rlib = libs
    gc = abi.bind_create(glib)
    rc = abi.bind_create(rlib)
    gid = _hit_world(gc)
    rid = _hit_world(rc)
    g = m3.World(gid)
    hits = 0
    for s in range(120):
        glib.m3World_Step(gid, C.c_float(DT), 4)
        rlib.m3World_Step(rid, C.c_float(DT), 4)
        want = _compare(glib, rlib, gid, rid, f"step {s + 1}")
        hits += len(want["m3World_HitEvents"])
    assert hits > 0
    assert g.hash() == rlib.m3World_Hash(rid)
    glib.m3DestroyWorld(gid)
    rlib.m3DestroyWorld(rid)
