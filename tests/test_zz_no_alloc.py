"""The allocation-free step entry point (needs a B200).

m3gpu_step_world_noalloc serves callers that may not allocate device
memory when they step (deadline-bound frame loops, code inside CUDA
graph capture, hosts whose device memory belongs to their own pool):
it steps an already-resident world with its scratch in a fixed device
array.  Its result must equal the regular entry point's bit for bit,
call after call.  This file runs last, alone or after the others.
"""
import ctypes as C

import pytest

from conftest import cuda_available
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
