"""Joint drives and switches (joint.h:183-248; joint.c:548-624,
732-1129) on the host: limits, motor, collide-connected, spring and drive
targets on revolute chains and fixed welds, with valid and refused
values, leave the world with the reference's hash, getters and journal
bytes; the reference's journal of them replays here to the same world,
and hostile records are refused whole as the reference's replay refuses
them (world.c:3050-3179)."""
import ctypes as C
import struct

from maul3d_b200 import abi
from maul3d_b200.abi import SCENE_TOWERS, SCENE_UNEVEN

Q = abi.m3Quat


def _commands(lib, wid):
    w0 = wid.index1 - 1
    j = [abi.m3JointId(k, w0, 0) for k in range(12)]
    lib.m3Joint_SetLimits(j[1], True, -0.5, 0.75)
    lib.m3Joint_SetLimits(j[2], True, 0.5, -0.5)                     # refused: unordered
    lib.m3Joint_SetLimits(j[3], False, float("nan"), 1.0)            # refused
    lib.m3Joint_SetMotor(j[2], True, 1.5, 40.0)
    lib.m3Joint_SetMotor(j[4], True, 1.5, -1.0)                      # refused
    lib.m3Joint_SetCollideConnected(j[5], True)
    lib.m3Joint_SetCollideConnected(j[6], False)
    lib.m3Joint_SetSpring(j[7], True, 4.0, 0.7)
    lib.m3Joint_SetSpring(j[8], True, 0.0, 0.7)                      # refused
    lib.m3Joint_SetSpring(j[8], True, 3.0, -0.1)                     # refused
    lib.m3Joint_SetTargetAngle(j[7], 0.4)
    lib.m3Joint_SetTargetAngle(j[9], 4.0)                            # refused: beyond pi
    lib.m3Joint_SetTargetTranslation(j[9], 0.5)                      # not prismatic
    lib.m3Joint_SetTargetRotation(j[10], Q(0.0, 0.0, 0.0, 1.0))      # not spherical
    lib.m3Joint_SetLimits(j[11], True, -0.25, 0.25)
    lib.m3Joint_SetLimits(j[11], False, -0.25, 0.25)
    stale = abi.m3JointId(3, w0, 9)
    lib.m3Joint_SetMotor(stale, True, 1.0, 1.0)
    lib.m3Joint_SetCollideConnected(stale, True)


def _getters(lib, wid):
    w0 = wid.index1 - 1
    rows = []
    for k in list(range(1, 14)) + [-3]:
        j = abi.m3JointId(abs(k), w0, 0 if k > 0 else 9)
        rows.append((lib.m3Joint_GetCollideConnected(j), lib.m3Joint_GetAngle(j),
                     lib.m3Joint_GetTranslation(j)))
    return rows


def _engines(m3, oracle):
    g = abi.bind_snapshot(abi.bind_joint_commands(m3.lib))
    r = abi.bind_snapshot(abi.bind_joint_commands(oracle.lib()))
    return g, r


def _journal(lib, wid, action):
    buf = (C.c_uint8 * 8192)()
    assert lib.m3World_JournalBegin(wid, buf, 8192)
    action()
    n = lib.m3World_JournalEnd(wid)
    assert n >= 0
    return bytes(buf[:n])


def _without_world_index(journal: bytes) -> bytes:
    out = bytearray(journal)
    cursor = 0
    while cursor < len(out):
        op, n = struct.unpack_from("<ii", out, cursor)
        out[cursor + 12:cursor + 14] = b"\0\0"
        cursor += 8 + n
    return bytes(out)


def test_joint_commands_match_the_reference(m3, oracle):
    glib, rlib = _engines(m3, oracle)
    for scene, seed, param in ((SCENE_UNEVEN, 51, 60), (SCENE_TOWERS, 52, 2)):
        g = m3.World.scene(scene, seed, param)
        r = oracle.RefWorld.scene(scene, seed, param)
        gj = _journal(glib, g.id, lambda: _commands(glib, g.id))
        rj = _journal(rlib, r.id, lambda: _commands(rlib, r.id))
        assert _without_world_index(gj) == _without_world_index(rj) and len(rj) > 0
        assert g.hash() == r.hash()
        assert _getters(glib, g.id) == _getters(rlib, r.id)
        g.destroy()
        r.destroy()


def test_reference_journal_of_joint_commands_replays_here(m3, oracle):
    glib, rlib = _engines(m3, oracle)
    r = oracle.RefWorld.scene(SCENE_UNEVEN, 53, 60)
    journal = _journal(rlib, r.id, lambda: _commands(rlib, r.id))
    g = m3.World.scene(SCENE_UNEVEN, 53, 60)
    buf = (C.c_uint8 * len(journal)).from_buffer_copy(journal)
    assert glib.m3World_JournalReplay(g.id, buf, len(journal))
    assert g.hash() == r.hash()
    assert _getters(glib, g.id) == _getters(rlib, r.id)
    r.destroy()
    g.destroy()


def test_hostile_joint_records_are_refused_whole(m3, oracle):
    glib, rlib = _engines(m3, oracle)
    g = m3.World.scene(SCENE_UNEVEN, 54, 60)
    r = oracle.RefWorld.scene(SCENE_UNEVEN, 54, 60)
    before = g.hash()
    w0 = g.id.index1 - 1
    joint = bytes(abi.m3JointId(2, w0, 0))
    stale = bytes(abi.m3JointId(2, w0, 5))
    good = abi.journal_record(54, joint + struct.pack("<i", 1))
    for bad in (abi.journal_record(52, joint + struct.pack("<iff", 1, 0.5, -0.5)),
                abi.journal_record(52, joint + struct.pack("<iff", 1, float("nan"), 0.5)),
                abi.journal_record(53, stale + struct.pack("<iff", 1, 1.0, 2.0)),
                abi.journal_record(53, joint + struct.pack("<if", 1, 1.0)),
                abi.journal_record(54, stale + struct.pack("<i", 1)),
                abi.journal_record(56, joint + struct.pack("<iff", 1, 0.0, 0.5)),
                abi.journal_record(56, joint + struct.pack("<iff", 1, 2.0, -0.5)),
                abi.journal_record(57, joint + struct.pack("<f4f", 0.5, float("inf"), 0, 0, 1)),
                abi.journal_record(57, joint + struct.pack("<f3f", 0.5, 0, 0, 1))):
        stream = good + bad
        gbuf = (C.c_uint8 * len(stream)).from_buffer_copy(stream)
        assert not glib.m3World_JournalReplay(g.id, gbuf, len(stream))
        assert g.hash() == before
        rbuf = (C.c_uint8 * len(stream)).from_buffer_copy(stream)
        assert not rlib.m3World_JournalReplay(r.id, rbuf, len(stream))
    g.destroy()
    r.destroy()
