"""Bit-exact parity of the device step (needs a B200).

The device path must produce the reference's world hash (FNV-1a over
bodies, shapes, joints, pair keys and the 188-byte manifolds) after
every step: against the committed golden traces (generated by the
oracle, tests/golden/make_golden.py), and step by step against the
oracle itself where its prebuilt library is present.  Integer and
byte state is compared exactly: the tolerance is zero.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import GOLDEN_CASES, cuda_available
from maul3d_b200.abi import (SCENE_BOX_PYRAMID, SCENE_FREEFALL, SCENE_SPHERE_PYRAMID, SCENE_TOWERS,
                             SCENE_UNEVEN)

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


@pytest.mark.parametrize("idx", range(GOLDEN_CASES))
def test_golden_trace_on_device(m3, golden, idx):
    case = golden["cases"][idx]
    w = m3.World.scene(case["scene"], case["seed"], case["param"])
    assert f"{w.hash():016x}" == case["hash0"]
    done = 0
    for step in sorted(int(s) for s in case["hashes"]):
        w.step(case["dt"], case["substeps"], step - done)
        done = step
        assert f"{w.hash():016x}" == case["hashes"][str(step)], f"{case['name']} step {step}"
    w.destroy()


def test_sphere_pyramid_reaches_reference_bench_pin(m3):
    # bench/pins.txt:1 of the reference: "pyramid 975f319f2f44cc5d".
    w = m3.World.scene(SCENE_SPHERE_PYRAMID)
    w.step(1.0 / 60.0, 4, 300)
    assert f"{w.hash():016x}" == "975f319f2f44cc5d"


@pytest.mark.parametrize("scene,seed,param,steps", [
    (SCENE_FREEFALL, 0, 8, 20),
    (SCENE_BOX_PYRAMID, 0, 20, 120),
    (SCENE_UNEVEN, 11, 48, 150),
    (SCENE_UNEVEN, 12, 300, 100),
    (SCENE_TOWERS, 7, 4, 120),
    (SCENE_TOWERS, 9, 24, 90),
])
def test_every_step_matches_oracle(m3, oracle, scene, seed, param, steps):
    g = m3.World.scene(scene, seed, param)
    r = oracle.RefWorld.scene(scene, seed, param)
    for s in range(steps):
        r.step(1.0 / 60.0, 4, 1)
        g.step(1.0 / 60.0, 4, 1)
        if g.hash() != r.hash():
            pytest.fail(f"step {s + 1}: {g.state().first_difference(r.state())}")
    assert g.state().first_difference(r.state()) is None


def test_batched_step_equals_worlds_stepped_alone(m3, oracle):
    sizes = [32, 40, 77, 128, 256, 33, 512, 64]
    batch = [m3.World.scene(SCENE_UNEVEN, 100 + i, n) for i, n in enumerate(sizes)]
    alone = [m3.World.scene(SCENE_UNEVEN, 100 + i, n) for i, n in enumerate(sizes)]
    m3.step_worlds(batch, 1.0 / 60.0, 4, 40)
    for w in alone:
        w.step(1.0 / 60.0, 4, 40)
    hb = m3.hash_worlds(batch)
    ha = np.array([w.hash() for w in alone], dtype=np.uint64)
    assert np.array_equal(hb, ha)
    refs = []
    for i, n in enumerate(sizes):
        r = oracle.RefWorld.scene(SCENE_UNEVEN, 100 + i, n)
        r.step(1.0 / 60.0, 4, 40)
        refs.append(r.hash())
    assert [int(h) for h in hb] == refs


def test_device_hash_equals_host_hash(m3):
    w = m3.World.scene(SCENE_UNEVEN, 3, 200)
    w.step(1.0 / 60.0, 4, 25)
    dev = int(m3.hash_worlds([w])[0])
    w.state()  # bring the host image up to date: the next hash runs on the host
    assert w.hash() == dev


def test_unsupported_feature_fails_loudly(m3):
    # Rolling resistance on a contact with a static body: the reference
    # writes the static body's spin (solver.c:542-545); the device path
    # refuses the world instead of racing on it.
    from maul3d_b200 import abi
    lib = abi.bind_create(m3.lib)
    wd = lib.m3DefaultWorldDef()
    wid = lib.m3CreateWorld(C.byref(wd))
    gd = lib.m3DefaultBodyDef()
    ground = lib.m3CreateBody(wid, C.byref(gd))
    sd = lib.m3DefaultShapeDef()
    sd.rollingResistance = 0.1
    plane = abi.m3Plane(abi.m3Vec3(0.0, 1.0, 0.0), 0.0)
    lib.m3CreatePlaneShape(ground, C.byref(sd), C.byref(plane))
    bd = lib.m3DefaultBodyDef()
    bd.type = 2
    bd.position = abi.m3Pos3(0.0, 0.49, 0.0)
    ball = lib.m3CreateBody(wid, C.byref(bd))
    sphere = abi.m3Sphere(abi.m3Vec3(0.0, 0.0, 0.0), 0.5)
    lib.m3CreateSphereShape(ball, C.byref(sd), C.byref(sphere))
    w = m3.World(wid)
    with pytest.raises(m3.M3GpuError) as err:
        w.step()
    assert err.value.code == m3.M3GPU_ERR_UNSUPPORTED
    # The world stays failed: every later step reports the refusal.
    with pytest.raises(m3.M3GpuError):
        w.step()


def _joint_ids(lib, world, count):
    from maul3d_b200 import abi
    w0 = world.id.index1 - 1
    return [bool(lib.m3Joint_IsValid(abi.m3JointId(j + 1, w0, 0))) for j in range(count)]


def test_broken_joint_slots_recycle_like_the_reference(m3, oracle):
    # Towers of welded boxes hit by dense spheres: the step destroys the
    # joints whose reaction passes their threshold (solver.c:4228-4257),
    # in ascending order, and a joint created afterwards takes the first
    # freed slot with its generation bumped (allocator.c:178-218).
    from maul3d_b200 import abi
    glib = abi.bind_create(m3.lib)
    rlib = abi.bind_create(oracle.lib())
    g = m3.World.scene(SCENE_TOWERS, 7, 4)
    r = oracle.RefWorld.scene(SCENE_TOWERS, 7, 4)
    for s in range(40):
        g.step(1.0 / 60.0, 4, 1)
        r.step(1.0 / 60.0, 4, 1)
        assert g.hash() == r.hash(), f"step {s + 1}"
    alive_g = _joint_ids(glib, g, 112)
    alive_r = _joint_ids(rlib, r, 112)
    assert alive_g == alive_r
    assert 0 < sum(alive_g) < 112, "the scene must break some joints and keep others"
    made = []
    for lib, world in ((glib, g), (rlib, r)):
        ids = []
        w0 = world.id.index1 - 1
        for k in range(3):
            jd = lib.m3DefaultJointDef()
            jd.type = 3
            jd.bodyA = abi.m3BodyId(2 + 4 * k, w0, 0)
            jd.bodyB = abi.m3BodyId(3 + 4 * k, w0, 0)
            jd.localAnchorA = abi.m3Vec3(0.5, 0.0, 0.0)
            jd.localAnchorB = abi.m3Vec3(-0.5, 0.0, 0.0)
            j = lib.m3CreateJoint(C.byref(jd))
            lib.m3Joint_SetBreakThresholds(j, 800.0, 0.0)
            ids.append((j.index1, j.generation))
        made.append(ids)
    assert made[0] == made[1]
    assert all(gen == 1 for _, gen in made[0]), made[0]
    assert g.hash() == r.hash()
    for s in range(60):
        g.step(1.0 / 60.0, 4, 1)
        r.step(1.0 / 60.0, 4, 1)
        if g.hash() != r.hash():
            pytest.fail(f"step {s + 41}: {g.state().first_difference(r.state())}")
