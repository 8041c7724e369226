"""Creation-time parity (CPU): worlds built through this library's
drop-in creation API hash bit-identically to the same worlds built by
the reference, and the mass properties, inertia tensors, extents and
interned hulls match byte for byte.  Also the reference's refusal
contract: bad input returns null ids and an error code, never a crash.
"""
import ctypes as C

import numpy as np
import pytest

from maul3d_b200.abi import (SCENE_BOX_PYRAMID, SCENE_FREEFALL, SCENE_MIXED,
                             SCENE_SPHERE_PYRAMID, SCENE_UNEVEN)

SCENES = [
    (SCENE_SPHERE_PYRAMID, 0, 0),
    (SCENE_BOX_PYRAMID, 0, 20),
    (SCENE_FREEFALL, 0, 8),
    (SCENE_UNEVEN, 1, 32),
    (SCENE_UNEVEN, 7, 600),
    (SCENE_UNEVEN, 5, 2048),
    (SCENE_MIXED, 3, 200),
    (SCENE_MIXED, 8, 1500),
]


@pytest.mark.parametrize("scene,seed,param", SCENES)
def test_world_hash_at_creation_matches_reference(m3, oracle, scene, seed, param):
    g = m3.World.scene(scene, seed, param)
    r = oracle.RefWorld.scene(scene, seed, param)
    assert g.body_count() == r.body_count()
    assert g.hash() == r.hash()
    gm, rm = g.mass(), r.mass()
    for key in gm:
        assert gm[key].tobytes() == rm[key].tobytes(), key
    g.destroy()
    r.destroy()


def test_hash64_is_fnv1a(m3, oracle):
    data = np.arange(97, dtype=np.uint8)
    for lib in (m3.lib, oracle.lib()):
        h = lib.m3Hash64(0xCBF29CE484222325, data.ctypes.data, len(data))
        expected = 0xCBF29CE484222325
        for b in data.tobytes():
            expected = ((expected ^ b) * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
        assert h == expected


def test_version_matches_reference(m3, oracle):
    assert m3.lib.m3GetVersion() == oracle.lib().m3GetVersion()


def test_refusals_return_null_ids(m3):
    lib = m3.lib
    from maul3d_b200.abi import m3WorldId
    # A stale world id: step is a no-op reported as invalid, hash is 0.
    stale = m3WorldId(60000, 7)
    lib.m3World_Step(stale, C.c_float(1.0 / 60.0), 4)
    assert m3.last_error()[0] == m3.M3GPU_ERR_INVALID
    assert lib.m3World_Hash(stale) == 0
    # Invalid dt and substeps on a live world are refused before any work.
    w = m3.World.scene(SCENE_FREEFALL, 0, 2)
    h = w.hash()
    lib.m3World_Step(w.id, C.c_float(0.0), 4)
    assert m3.last_error()[0] == m3.M3GPU_ERR_INVALID
    lib.m3World_Step(w.id, C.c_float(1.0 / 60.0), 257)
    assert m3.last_error()[0] == m3.M3GPU_ERR_INVALID
    assert w.hash() == h
    w.destroy()
    assert not lib.m3World_IsValid(w.id)


def test_unknown_scene_is_null(m3):
    with pytest.raises(m3.M3GpuError):
        m3.World.scene(99)


@pytest.mark.parametrize("scene,seed,param", SCENES[:4])
def test_counters_at_creation_match_reference(m3, oracle, scene, seed, param):
    """m3World_GetCounters on a freshly built world: the live counts, the
    tree height and the snapshot size equal the reference's (the scratch
    and allocation figures are engine-specific)."""
    g = m3.World.scene(scene, seed, param)
    r = oracle.RefWorld.scene(scene, seed, param)
    gc = m3.counters(g)
    rc = oracle.lib().m3World_GetCounters(r.id)
    for name in ("bodyCount", "shapeCount", "jointCount", "contactCount", "awakeCount",
                 "islandCount", "colorCount", "hullCount", "meshCount", "treeHeight",
                 "snapshotBytes"):
        assert gc[name] == getattr(rc, name), name
    assert m3.profile(g)["step"] == 0.0
    g.destroy()
    r.destroy()
