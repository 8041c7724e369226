"""Snapshot restore and journal ingestion (CPU): a snapshot the reference
engine takes (format v54, snapshot.c:613-678) restores into a world of
this library with the reference's hash, pools and free queues; corrupt,
foreign or unsupported snapshots are refused with the world untouched
(snapshot.c:680-826).  Journal records of body commands apply with the
reference's arithmetic (body.c:351-418, world.c:2283-2321); stepping
journals run on the GPU (tests/test_serving_gpu.py).
"""
import ctypes as C
import struct

import numpy as np
import pytest

from maul3d_b200 import abi
from maul3d_b200.abi import SCENE_BOX_PYRAMID, SCENE_TOWERS, SCENE_UNEVEN


def _snapshot(lib, wid) -> bytes:
    n = lib.m3World_SnapshotSize(wid)
    assert n > 0
    buf = (C.c_uint8 * n)()
    assert lib.m3World_Snapshot(wid, buf, n) == n
    return bytes(buf)


def _restore(lib, wid, data: bytes) -> bool:
    buf = (C.c_uint8 * len(data)).from_buffer_copy(data)
    return bool(lib.m3World_Restore(wid, buf, len(data)))


def _replay(lib, wid, data: bytes) -> bool:
    buf = (C.c_uint8 * max(len(data), 1)).from_buffer_copy(data or b"\0")
    return bool(lib.m3World_JournalReplay(wid, buf, len(data)))


@pytest.fixture(scope="module")
def libs(m3, oracle):
    ref = abi.bind_snapshot(abi.bind_create(oracle.lib()))
    ours = abi.bind_snapshot(abi.bind_create(m3.lib))
    return ours, ref


@pytest.mark.parametrize("scene,seed,param,steps", [
    (SCENE_BOX_PYRAMID, 0, 20, 40),
    (SCENE_UNEVEN, 21, 64, 90),
    (SCENE_TOWERS, 7, 4, 40),
])
def test_reference_snapshot_restores_with_the_reference_hash(m3, oracle, libs, scene, seed,
                                                            param, steps):
    ours, ref = libs
    r = oracle.RefWorld.scene(scene, seed, param)
    r.step(1.0 / 60.0, 4, steps)
    snap = _snapshot(ref, r.id)
    # A fresh world of the same scene (same capacities), never stepped.
    g = m3.World.scene(scene, seed, param)
    assert _restore(ours, g.id, snap), m3.last_error()
    assert g.hash() == r.hash()
    assert g.state().first_difference(r.state()) is None
    g.destroy()
    r.destroy()


def test_restore_recycles_slots_like_the_reference(m3, oracle, libs):
    # Joints broken before the snapshot sit in its free queue: a joint
    # created after the restore takes the first one, with its generation.
    ours, ref = libs
    r = oracle.RefWorld.scene(SCENE_TOWERS, 7, 4)
    r.step(1.0 / 60.0, 4, 40)
    snap = _snapshot(ref, r.id)
    g = m3.World.scene(SCENE_TOWERS, 7, 4)
    assert _restore(ours, g.id, snap)
    made = []
    for lib, wid in ((ours, g.id), (ref, r.id)):
        jd = lib.m3DefaultJointDef()
        jd.type = 3
        jd.bodyA = abi.m3BodyId(2, wid.index1 - 1, 0)
        jd.bodyB = abi.m3BodyId(3, wid.index1 - 1, 0)
        jd.localAnchorA = abi.m3Vec3(0.5, 0.0, 0.0)
        jd.localAnchorB = abi.m3Vec3(-0.5, 0.0, 0.0)
        j = lib.m3CreateJoint(C.byref(jd))
        made.append((j.index1, j.generation))
    assert made[0] == made[1] and made[0][1] == 1
    assert g.hash() == r.hash()


def test_corrupt_or_foreign_snapshots_are_refused_untouched(m3, oracle, libs):
    ours, ref = libs
    r = oracle.RefWorld.scene(SCENE_UNEVEN, 3, 48)
    r.step(1.0 / 60.0, 4, 10)
    snap = _snapshot(ref, r.id)
    g = m3.World.scene(SCENE_UNEVEN, 4, 48)
    before = g.hash()
    bad_magic = b"X" + snap[1:]
    assert not _restore(ours, g.id, bad_magic)
    assert not _restore(ours, g.id, snap[:-1])
    assert not _restore(ours, g.id, snap + b"\0")
    # A flipped pool cursor (body maxIndex beyond capacity).
    cur = bytearray(snap)
    cur[28:32] = (10 ** 6).to_bytes(4, "little")
    assert not _restore(ours, g.id, bytes(cur))
    assert m3.last_error()[0] == m3.M3GPU_ERR_INVALID
    assert g.hash() == before
    # A world of other capacities.
    other = m3.World.scene(SCENE_UNEVEN, 3, 64)
    assert not _restore(ours, other.id, snap)
    # The same bytes restore fine into the right world.
    assert _restore(ours, g.id, snap)
    assert g.hash() == r.hash()


class _WaterVolumeDef(C.Structure):
    # world.h:107-116 of the reference.
    _fields_ = [("lo", abi.m3Pos3), ("hi", abi.m3Pos3), ("density", C.c_float),
                ("linearDrag", C.c_float), ("angularDrag", C.c_float), ("flow", abi.m3Vec3),
                ("internalValue", C.c_int32)]


class _WaterVolumeId(C.Structure):
    _fields_ = [("index1", C.c_int32), ("world0", C.c_uint16), ("generation", C.c_uint16)]


def test_unmodelled_content_is_refused(m3, oracle, libs):
    # A live water volume (a pool this path does not model) in the
    # snapshot: refused as unsupported, the world untouched.
    ours, ref = libs
    lib = oracle.lib()
    lib.m3DefaultWaterVolumeDef.restype = _WaterVolumeDef
    lib.m3CreateWaterVolume.argtypes = [abi.m3WorldId, C.POINTER(_WaterVolumeDef)]
    lib.m3CreateWaterVolume.restype = _WaterVolumeId
    r = oracle.RefWorld.scene(SCENE_UNEVEN, 3, 48)
    wd = lib.m3DefaultWaterVolumeDef()
    wd.lo = abi.m3Pos3(-5.0, -1.0, -5.0)
    wd.hi = abi.m3Pos3(5.0, 0.5, 5.0)
    vol = lib.m3CreateWaterVolume(r.id, C.byref(wd))
    assert vol.index1 > 0
    snap = _snapshot(ref, r.id)
    g = m3.World.scene(SCENE_UNEVEN, 3, 48)
    before = g.hash()
    assert not _restore(ours, g.id, snap)
    assert m3.last_error()[0] == m3.M3GPU_ERR_UNSUPPORTED
    assert g.hash() == before


def test_body_commands_replay_like_the_reference(m3, oracle, libs):
    ours, ref = libs
    r = oracle.RefWorld.scene(SCENE_UNEVEN, 5, 64)
    r.step(1.0 / 60.0, 4, 20)
    snap = _snapshot(ref, r.id)
    g = m3.World.scene(SCENE_UNEVEN, 5, 64)
    assert _restore(ours, g.id, snap)
    rng = np.random.default_rng(5)
    journal = b""
    ops = [abi.OP_APPLY_LINEAR_IMPULSE, abi.OP_APPLY_ANGULAR_IMPULSE, abi.OP_APPLY_FORCE,
           abi.OP_APPLY_TORQUE, abi.OP_SET_LINEAR_VELOCITY, abi.OP_SET_ANGULAR_VELOCITY]
    for k in range(40):
        body = int(rng.integers(2, 60))
        v = [float(x) for x in rng.uniform(-50, 50, 3).astype(np.float32)]
        journal += abi.journal_body_command(ops[k % len(ops)], body, 0, v)
    assert _replay(ref, r.id, journal)
    assert _replay(ours, g.id, journal)
    assert g.hash() == r.hash()
    assert g.state().first_difference(r.state()) is None


def test_bad_or_unsupported_journals_are_refused_untouched(m3, libs):
    ours, _ = libs
    g = m3.World.scene(SCENE_UNEVEN, 5, 64)
    before = g.hash()
    good = abi.journal_body_command(abi.OP_APPLY_LINEAR_IMPULSE, 3, 0, [1.0, 2.0, 3.0])
    # Truncated, stale body, non-finite vector, unknown and unsupported ops.
    assert not _replay(ours, g.id, good + good[:-1])
    assert not _replay(ours, g.id, good + abi.journal_body_command(28, 9999, 0, [1, 1, 1]))
    assert not _replay(ours, g.id, good + abi.journal_body_command(28, 3, 0, [float("nan"), 0, 0]))
    assert not _replay(ours, g.id, good + abi.journal_step(0.0, 4))
    assert not _replay(ours, g.id, good + abi.journal_step(1 / 60, 300))
    unsupported = C.c_int32(61).value.to_bytes(4, "little") + (0).to_bytes(4, "little")
    assert not _replay(ours, g.id, good + unsupported)
    assert m3.last_error()[0] == m3.M3GPU_ERR_UNSUPPORTED
    assert g.hash() == before
    assert _replay(ours, g.id, good)
    assert g.hash() != before


@pytest.mark.parametrize("scene,seed,param", [
    (SCENE_BOX_PYRAMID, 0, 20),
    (SCENE_UNEVEN, 1, 32),
    (SCENE_UNEVEN, 7, 600),
    (SCENE_TOWERS, 7, 4),
])
def test_snapshot_of_a_new_world_is_the_references_bytes(m3, oracle, libs, scene, seed, param):
    # Every block, the broadphase tree built by the creation inserts
    # (dynamic_tree.c:221-322) and the id pools included.
    ours, ref = libs
    r = oracle.RefWorld.scene(scene, seed, param)
    g = m3.World.scene(scene, seed, param)
    assert ours.m3World_SnapshotSize(g.id) == ref.m3World_SnapshotSize(r.id)
    assert _snapshot(ours, g.id) == _snapshot(ref, r.id)


@pytest.mark.parametrize("scene,seed,param,steps", [
    (SCENE_UNEVEN, 21, 64, 90),
    (SCENE_TOWERS, 7, 4, 40),
])
def test_restored_world_snapshots_the_same_bytes(m3, oracle, libs, scene, seed, param, steps):
    # Restore then snapshot gives back the input byte for byte, the state
    # this path does not model included.
    ours, ref = libs
    r = oracle.RefWorld.scene(scene, seed, param)
    r.step(1.0 / 60.0, 4, steps)
    snap = _snapshot(ref, r.id)
    g = m3.World.scene(scene, seed, param)
    assert _restore(ours, g.id, snap)
    assert _snapshot(ours, g.id) == snap
    small = (C.c_uint8 * 16)()
    assert ours.m3World_Snapshot(g.id, small, 16) == -1


def _record_session(lib, wid, joints=()):
    """Body commands and joint thresholds on one world, recorded."""
    buf = (C.c_uint8 * 4096)()
    assert lib.m3World_JournalBegin(wid, buf, 4096)
    w0 = wid.index1 - 1
    for k in range(6):
        b = abi.m3BodyId(3 + k, w0, 0)
        lib.m3Body_ApplyLinearImpulse(b, abi.m3Vec3(1.5 * k, 2.0, -0.5))
        lib.m3Body_ApplyAngularImpulse(b, abi.m3Vec3(0.1, -0.2 * k, 0.3))
        lib.m3Body_SetLinearVelocity(b, abi.m3Vec3(0.0, 0.5 * k, 0.0))
        lib.m3Body_ApplyForce(b, abi.m3Vec3(3.0, 0.0, 1.0))
        lib.m3Body_ApplyTorque(b, abi.m3Vec3(0.0, 1.0, 0.0))
        lib.m3Body_SetAngularVelocity(b, abi.m3Vec3(0.2, 0.0, 0.1))
    lib.m3Body_ApplyLinearImpulse(abi.m3BodyId(1, w0, 0), abi.m3Vec3(1.0, 1.0, 1.0))  # static: no-op
    for j in joints:
        lib.m3Joint_SetBreakThresholds(abi.m3JointId(j, w0, 0), 300.0, 50.0)
    n = lib.m3World_JournalEnd(wid)
    assert n > 0
    return bytes(buf[:n])


def _without_world_index(journal: bytes) -> bytes:
    """The records with the recording world's index (the world0 half of
    every body or joint id, which replay retargets) cleared."""
    out = bytearray(journal)
    cursor = 0
    while cursor < len(out):
        op, n = struct.unpack_from("<ii", out, cursor)
        if op != abi.OP_STEP:
            out[cursor + 12:cursor + 14] = b"\0\0"
        cursor += 8 + n
    return bytes(out)


def test_recorded_journals_are_the_references_bytes(m3, oracle, libs):
    ours, ref = libs
    g = m3.World.scene(SCENE_TOWERS, 7, 2)
    r = oracle.RefWorld.scene(SCENE_TOWERS, 7, 2)
    a = _record_session(ours, g.id, joints=(1, 5, 9))
    b = _record_session(ref, r.id, joints=(1, 5, 9))
    assert _without_world_index(a) == _without_world_index(b)
    assert g.hash() == r.hash()
    # Our recording replays in the reference, and the reference's in ours.
    g2 = m3.World.scene(SCENE_TOWERS, 7, 2)
    r2 = oracle.RefWorld.scene(SCENE_TOWERS, 7, 2)
    assert _replay(ours, g2.id, b) and _replay(ref, r2.id, a)
    assert g2.hash() == r2.hash() == r.hash()


def test_creation_during_a_recording_ends_it_unrecordable(m3, libs):
    ours, _ = libs
    g = m3.World.scene(SCENE_UNEVEN, 1, 32)
    buf = (C.c_uint8 * 1024)()
    assert ours.m3World_JournalBegin(g.id, buf, 1024)
    assert not ours.m3World_JournalBegin(g.id, buf, 1024)  # one session at a time
    bd = ours.m3DefaultBodyDef()
    ours.m3CreateBody(g.id, C.byref(bd))
    assert ours.m3World_JournalEnd(g.id) == -1
    # Overflow ends a session the same way.
    small = (C.c_uint8 * 16)()
    assert ours.m3World_JournalBegin(g.id, small, 16)
    ours.m3Body_ApplyLinearImpulse(abi.m3BodyId(3, g.id.index1 - 1, 0), abi.m3Vec3(1.0, 0.0, 0.0))
    assert ours.m3World_JournalEnd(g.id) == -1


def _tree_blocks(snap: bytes):
    """(root, free list, proxy ids, nodes) of a snapshot: the header
    cursors and the blocks after the pair keys (snapshot.c:243-247)."""
    h = np.frombuffer(snap[:192], dtype=np.int32)
    body_cap, shape_cap = int(h[6]), int(h[11])
    per_body = 40 + 12 + 12 + 4 + 36 + 36 + 12 + 4 + 4 + 4 + 1 + 1 + 4 + 1 + 4 + 4 + 8 + 32 \
        + 12 + 12 + 1 + 1 + 4 + 1 + 1 + 40
    off = 192 + per_body * body_cap + 58 + (2 + 1 + 4 + 4) * body_cap
    off += (4 + 1 + 32 + 4 + 4 + 4 + 8 + 4 + 2 + 1 + 4) * shape_cap + 8 * 8 * shape_cap
    proxies = np.frombuffer(snap[off:off + 4 * shape_cap], dtype=np.int32)
    nodes = np.frombuffer(snap[off + 4 * shape_cap:off + 4 * shape_cap + 144 * shape_cap],
                          dtype=np.uint8).reshape(2 * shape_cap, 72)
    return int(h[17]), int(h[18]), proxies, nodes


def test_tree_moves_on_the_host_rebuild_the_references_tree(m3, oracle, libs):
    # Each reference step reinserts the leaves its shapes escaped, in
    # shape order (broad_phase.c:500-539).  Read those moves off two
    # consecutive reference snapshots and make them with this library's
    # tree code on the restored earlier one: the tree must come out as
    # the reference's, byte for byte (removals, insertions, rotations).
    ours, ref = libs
    m3.lib.m3gpu_tree_move.argtypes = [abi.m3WorldId, C.c_int32, C.c_void_p, C.c_void_p]
    m3.lib.m3gpu_tree_move.restype = C.c_int32
    r = oracle.RefWorld.scene(SCENE_UNEVEN, 9, 300)
    g = m3.World.scene(SCENE_UNEVEN, 9, 300)
    total = 0
    before = _snapshot(ref, r.id)
    for step in range(12):
        r.step(1.0 / 60.0, 4, 1)
        after = _snapshot(ref, r.id)
        _, _, p0, n0 = _tree_blocks(before)
        root1, free1, p1, n1 = _tree_blocks(after)
        assert _restore(ours, g.id, before)
        for shape in range(len(p1)):
            if p1[shape] < 0:
                continue
            old = n0[p0[shape]][:48].tobytes()
            new = n1[p1[shape]][:48].tobytes()
            if old != new or p0[shape] != p1[shape]:
                bounds = np.frombuffer(new, dtype=np.float64)
                lo = np.ascontiguousarray(bounds[:3])
                hi = np.ascontiguousarray(bounds[3:])
                assert m3.lib.m3gpu_tree_move(g.id, shape, lo.ctypes.data, hi.ctypes.data) >= 0
                total += 1
        root, free, p, n = _tree_blocks(_snapshot(ours, g.id))
        assert (root, free) == (root1, free1), f"step {step + 1}"
        assert np.array_equal(p, p1), f"step {step + 1}"
        assert np.array_equal(n, n1), f"step {step + 1}"
        before = after
    assert total > 100
