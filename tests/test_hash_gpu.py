"""The parallel device world hash (needs a B200).

The device hashes each world's byte stream with one thread block
(bit-plane rounds for the low byte of the FNV state, ordered affine
scans for the rest).  It must equal the sequential FNV-1a of the same
stream: the host's m3WorldHashView and the reference's own
m3World_Hash.  Exact equality; integer arithmetic throughout.
"""
import ctypes as C

import pytest

from conftest import cuda_available
from maul3d_b200.abi import SCENE_BOX_PYRAMID, SCENE_FREEFALL, SCENE_SPHERE_PYRAMID, SCENE_UNEVEN

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

# Stream lengths from a few hundred bytes (freefall) past one 64 KiB
# staging round and many 8 KiB tiles (uneven 2048).
CASES = [
    (SCENE_FREEFALL, 0, 1, 0),
    (SCENE_FREEFALL, 0, 8, 3),
    (SCENE_SPHERE_PYRAMID, 0, 0, 5),
    (SCENE_BOX_PYRAMID, 0, 4, 7),
    (SCENE_BOX_PYRAMID, 0, 20, 2),
    (SCENE_UNEVEN, 11, 32, 4),
    (SCENE_UNEVEN, 12, 300, 6),
    (SCENE_UNEVEN, 13, 2048, 3),
]


@pytest.mark.parametrize("scene,seed,param,steps", CASES)
def test_device_hash_equals_reference(m3, oracle, scene, seed, param, steps):
    g = m3.World.scene(scene, seed, param)
    r = oracle.RefWorld.scene(scene, seed, param)
    if steps:
        g.step(1.0 / 60.0, 4, steps)
        r.step(1.0 / 60.0, 4, steps)
    else:
        m3.upload_worlds([g])
    dev = int(m3.hash_worlds([g])[0])
    assert dev == r.hash()
    g.state()  # host image current again: the next hash folds on the host
    assert g.hash() == dev
    g.destroy()
    r.destroy()


def test_batched_device_hash_matches_each_world(m3, oracle):
    specs = [(SCENE_UNEVEN, 40 + k, n) for k, n in enumerate([32, 2048, 64, 700, 128, 33])]
    gs = [m3.World.scene(*s) for s in specs]
    rs = [oracle.RefWorld.scene(*s) for s in specs]
    m3.step_worlds(gs, 1.0 / 60.0, 4, 3)
    for r in rs:
        r.step(1.0 / 60.0, 4, 3)
    hashes = [int(h) for h in m3.hash_worlds(gs)]
    assert hashes == [r.hash() for r in rs]
    for w in gs + rs:
        w.destroy()


def test_empty_and_off_default_worlds(m3, oracle):
    """A world with no bodies (header and pair count only) and a world
    whose tuning knobs are off their defaults (the optional header
    block) hash like the reference's on the device."""
    from maul3d_b200 import abi
    glib = abi.bind_create(m3.lib)
    rlib = abi.bind_create(oracle.lib())
    for tune in (False, True):
        ids = []
        for lib in (glib, rlib):
            wd = lib.m3DefaultWorldDef()
            if tune:
                wd.contactHertz = 45.0
                wd.enableSleeping = 0
            wid = lib.m3CreateWorld(C.byref(wd))
            if tune:
                bd = lib.m3DefaultBodyDef()
                bd.type = 2
                bd.position = abi.m3Pos3(0.0, 2.0, 0.0)
                body = lib.m3CreateBody(wid, C.byref(bd))
                sd = lib.m3DefaultShapeDef()
                sphere = abi.m3Sphere(abi.m3Vec3(0.0, 0.0, 0.0), 0.5)
                lib.m3CreateSphereShape(body, C.byref(sd), C.byref(sphere))
            lib.m3World_Step(wid, C.c_float(1.0 / 60.0), 4)
            ids.append(wid)
        gw = m3.World(ids[0])
        dev = int(m3.hash_worlds([gw])[0])
        assert dev == rlib.m3World_Hash(ids[1])
        glib.m3DestroyWorld(ids[0])
        rlib.m3DestroyWorld(ids[1])
