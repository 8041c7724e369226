"""The allocation-free step entry point (needs a B200).

m3gpu_step_world_noalloc serves callers that may not allocate device
memory when they step (deadline-bound frame loops, where allocating can
stall the whole device; hosts whose device memory belongs to their own
pool): it steps an already-resident world with its scratch in a fixed
device array.  Its result must equal the regular entry point's bit for
bit, call after call.

The file is named to be collected last: the entry point shares one
static device array with every later call, so if it ever failed, a run
that stops at the first failure has already run every other test.  Each
test here stands alone: it passes in a fresh process and after the
others.
"""
import ctypes as C

import pytest

from conftest import cuda_available
from maul3d_b200 import abi
from maul3d_b200.abi import SCENE_BOX_PYRAMID, SCENE_SHOTS, SCENE_TERRAIN, SCENE_UNEVEN, m3WorldId

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


def _bind(m3):
    fn = m3.lib.m3gpu_step_world_noalloc
    fn.argtypes = [m3WorldId, C.c_float, C.c_int32]
    fn.restype = C.c_int32
    return fn


@pytest.mark.parametrize("scene,seed,param", [(SCENE_UNEVEN, 41, 200), (SCENE_UNEVEN, 42, 700),
                                              (SCENE_TERRAIN, 44, 60), (SCENE_SHOTS, 45, 24)])
def test_noalloc_step_equals_regular_step_twice(m3, scene, seed, param):
    step_noalloc = _bind(m3)
    regular = m3.World.scene(scene, seed, param)
    static = m3.World.scene(scene, seed, param)
    # Residency is set up beforehand, where allocating is allowed.
    m3.reserve_worlds([regular, static])
    m3.upload_worlds([regular, static])
    for _ in range(2):
        m3.step_worlds([regular], 1.0 / 60.0, 4, 1)
        rc = step_noalloc(static.id, 1.0 / 60.0, 4)
        assert rc == m3.M3GPU_OK, m3.last_error()
        # Exact equality: the hash covers every body, pair and manifold byte.
        assert int(m3.hash_worlds([static])[0]) == int(m3.hash_worlds([regular])[0])
    assert static.state().first_difference(regular.state()) is None
    regular.destroy()
    static.destroy()


def test_noalloc_refuses_oversize_and_nonresident_worlds(m3):
    step_noalloc = _bind(m3)
    big = m3.World.scene(SCENE_BOX_PYRAMID, 0, 20)  # default capacities: 2048 shape slots
    m3.reserve_worlds([big])
    m3.upload_worlds([big])
    h = int(m3.hash_worlds([big])[0])
    assert step_noalloc(big.id, 1.0 / 60.0, 4) == m3.M3GPU_ERR_CAPACITY
    assert "allocation-free step holds" in m3.last_error()[1]
    assert int(m3.hash_worlds([big])[0]) == h
    fresh = m3.World.scene(SCENE_UNEVEN, 43, 64)  # built on the host, never uploaded
    assert step_noalloc(fresh.id, 1.0 / 60.0, 4) == m3.M3GPU_ERR_INVALID
    assert "not resident" in m3.last_error()[1]
    big.destroy()
    fresh.destroy()


def _seventeen_planes(m3):
    """A small world the device refuses (more than 16 planes), with
    capacities that fit the allocation-free scratch."""
    lib = abi.bind_create(m3.lib)
    wd = lib.m3DefaultWorldDef()
    wd.bodyCapacity = 16
    wd.shapeCapacity = 32
    wd.jointCapacity = 4
    wid = lib.m3CreateWorld(C.byref(wd))
    ground = lib.m3CreateBody(wid, C.byref(lib.m3DefaultBodyDef()))
    sd = lib.m3DefaultShapeDef()
    for k in range(17):
        plane = abi.m3Plane(abi.m3Vec3(0.0, 1.0, 0.0), -0.25 * k)
        lib.m3CreatePlaneShape(ground, C.byref(sd), C.byref(plane))
    for k in range(3):
        bd = lib.m3DefaultBodyDef()
        bd.type = 2
        bd.position = abi.m3Pos3(1.5 * k, 2.0, 0.0)
        body = lib.m3CreateBody(wid, C.byref(bd))
        ball = abi.m3Sphere(abi.m3Vec3(0.0, 0.0, 0.0), 0.5)
        lib.m3CreateSphereShape(body, C.byref(sd), C.byref(ball))
    return m3.World(wid)


def test_noalloc_refused_world_leaves_its_tree_and_the_next_world_alone(m3):
    """A world refused inside the step (here: 17 planes) after another
    world filled the shared scratch with its tree moves: the refusal is
    reported, the refused world's snapshot bytes (its broadphase tree
    included) do not change, a second call stays refused, and the first
    world still steps exactly like the regular entry point."""
    step_noalloc = _bind(m3)
    tracked = m3.World.scene(SCENE_UNEVEN, 46, 120)
    regular = m3.World.scene(SCENE_UNEVEN, 46, 120)
    planes = _seventeen_planes(m3)
    m3.reserve_worlds([tracked, regular, planes])
    m3.upload_worlds([tracked, regular, planes])
    for _ in range(2):
        assert step_noalloc(tracked.id, 1.0 / 60.0, 4) == m3.M3GPU_OK, m3.last_error()
        m3.step_worlds([regular], 1.0 / 60.0, 4, 1)
    before = m3.snapshot(planes)
    for _ in range(2):
        assert step_noalloc(planes.id, 1.0 / 60.0, 4) == m3.M3GPU_ERR_UNSUPPORTED
        assert "stalled" in m3.last_error()[1]
        assert m3.snapshot(planes) == before
    assert step_noalloc(tracked.id, 1.0 / 60.0, 4) == m3.M3GPU_OK, m3.last_error()
    m3.step_worlds([regular], 1.0 / 60.0, 4, 1)
    assert int(m3.hash_worlds([tracked])[0]) == int(m3.hash_worlds([regular])[0])
    assert m3.snapshot(tracked) == m3.snapshot(regular)
    for w in (tracked, regular, planes):
        w.destroy()
