"""Device snapshot slots (GPU): a world saved into an HBM slot, stepped
on, restored and stepped again repeats its own trace and the reference's
uninterrupted run, hash for hash, through revolute chains, joint
breakage and slot recycling, 16-point hulls and heightfields; its
snapshot bytes after the restore equal the reference's; a slot is void
once the world is built on.  CPU: the entry points refuse without a
device and for bad arguments.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import cuda_available
from maul3d_b200 import abi
from maul3d_b200.abi import SCENE_MIXED, SCENE_TERRAIN, SCENE_TOWERS, SCENE_UNEVEN

DT, SUB = 1.0 / 60.0, 4


def _trace(m3, w, steps):
    out = []
    for _ in range(steps):
        m3.step_worlds([w], DT, SUB, 1)
        out.append(w.hash())
    return out


def test_slot_calls_refuse_bad_arguments(m3):
    w = m3.World.scene(SCENE_UNEVEN, 1, 40)
    assert m3.lib.m3gpu_slots_reserve(w.id, -1) == m3.M3GPU_ERR_INVALID
    assert m3.lib.m3gpu_slot_save(w.id, 0) == m3.M3GPU_ERR_INVALID  # no slots reserved
    assert m3.lib.m3gpu_slot_restore(w.id, 3) == m3.M3GPU_ERR_INVALID
    w.destroy()
    assert m3.lib.m3gpu_slot_save(w.id, 0) == m3.M3GPU_ERR_INVALID  # stale world


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")
@pytest.mark.parametrize("scene,seed,param", [
    (SCENE_UNEVEN, 3, 300),
    (SCENE_TOWERS, 7, 6),
    (SCENE_MIXED, 4, 400),
    (SCENE_TERRAIN, 2, 120),
])
def test_restored_slots_repeat_the_reference_run(m3, oracle, scene, seed, param):
    r = oracle.RefWorld.scene(scene, seed, param)
    ref = [int(h) for h in r.trace(DT, SUB, 60)]
    r.destroy()
    w = m3.World.scene(scene, seed, param)
    w.reserve_slots(4)
    got = _trace(m3, w, 10)
    w.save_slot(0)                     # after step 10
    got += _trace(m3, w, 15)
    w.save_slot(1)                     # after step 25
    got += _trace(m3, w, 35)
    assert got == ref
    # Back to step 10: the next 50 steps again, with a save on the way.
    w.restore_slot(0)
    again = _trace(m3, w, 20)
    w.save_slot(2)                     # after step 30
    again += _trace(m3, w, 30)
    assert again == ref[10:60]
    # Back to step 25, then to step 30.
    w.restore_slot(1)
    assert _trace(m3, w, 5) == ref[25:30]
    w.restore_slot(2)
    assert _trace(m3, w, 10) == ref[30:40]
    w.destroy()


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")
def test_snapshot_after_a_restored_slot_equals_the_reference(m3, oracle):
    # Joint breakage drains freed joint slots into the host's free queue
    # on every readback: a restore brings that queue back with the device
    # state, so the snapshot (pools, free queues, tree) matches.
    r = oracle.RefWorld.scene(SCENE_TOWERS, 11, 6)
    r.step(DT, SUB, 40)
    lib = abi.bind_snapshot(abi.bind_create(oracle.lib()))
    n = lib.m3World_SnapshotSize(r.id)
    buf = (C.c_uint8 * n)()
    assert lib.m3World_Snapshot(r.id, buf, n) == n
    expected = bytes(buf)
    r.destroy()
    w = m3.World.scene(SCENE_TOWERS, 11, 6)
    w.reserve_slots(1)
    m3.step_worlds([w], DT, SUB, 10)
    w.save_slot(0)
    m3.step_worlds([w], DT, SUB, 50)
    w.hash()
    m3.snapshot(w)                     # readbacks drain broken joints on the host
    w.restore_slot(0)
    m3.step_worlds([w], DT, SUB, 30)
    assert m3.snapshot(w) == expected
    w.destroy()


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")
def test_a_slot_is_void_once_the_world_is_built_on(m3):
    w = m3.World.scene(SCENE_UNEVEN, 5, 64)
    w.reserve_slots(2)
    m3.step_worlds([w], DT, SUB, 3)
    w.save_slot(0)
    lib = abi.bind_create(m3.lib)
    bd = lib.m3DefaultBodyDef()
    bd.type = 2
    bd.position = abi.m3Pos3(0.0, 30.0, 0.0)
    assert lib.m3CreateBody(w.id, C.byref(bd)).index1 > 0
    with pytest.raises(m3.M3GpuError):
        w.restore_slot(0)
    with pytest.raises(m3.M3GpuError):
        w.restore_slot(1)              # never saved
    w.destroy()


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")
def test_device_body_commands_equal_the_reference_body_calls(m3, oracle):
    # Every command kind on random bodies, plus the no-ops: the static
    # ground (impulses need mass), a stale id, a non-finite vector.
    rlib = abi.bind_create(oracle.lib())
    r = oracle.RefWorld.scene(SCENE_MIXED, 9, 300)
    w = m3.World.scene(SCENE_MIXED, 9, 300)
    bodies = w.body_count()
    names = {abi.OP_APPLY_LINEAR_IMPULSE: "m3Body_ApplyLinearImpulse",
             29: "m3Body_ApplyAngularImpulse", 26: "m3Body_ApplyForce", 27: "m3Body_ApplyTorque",
             4: "m3Body_SetLinearVelocity", 5: "m3Body_SetAngularVelocity"}
    ops = sorted(names)
    rng = np.random.default_rng(4)
    for step in range(30):
        cmds = []
        for _ in range(int(rng.integers(0, 9))):
            op = ops[int(rng.integers(0, len(ops)))]
            index1 = int(rng.integers(1, bodies + 1))
            v = tuple(float(x) for x in rng.normal(size=3).astype(np.float32) * 5.0)
            cmds.append((op, index1, 0, v))
        if step == 7:
            cmds.append((abi.OP_APPLY_LINEAR_IMPULSE, 1, 0, (0.0, 9.0, 0.0)))      # static ground
            cmds.append((abi.OP_APPLY_LINEAR_IMPULSE, 100000, 0, (0.0, 9.0, 0.0)))  # stale
            cmds.append((4, 3, 0, (float("nan"), 0.0, 0.0)))                       # non-finite
        for op, index1, gen, v in cmds:
            getattr(rlib, names[op])(abi.m3BodyId(index1, r.id.index1 - 1, gen), abi.m3Vec3(*v))
        r.step(DT, SUB, 1)
        m3.step_worlds_commands([w], [(0, op, abi.m3BodyId(index1, w.id.index1 - 1, gen), v)
                                      for op, index1, gen, v in cmds], DT, SUB)
        assert w.hash() == r.hash(), f"step {step}"
    r.destroy()
    w.destroy()
