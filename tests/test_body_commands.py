"""Body commands at a world point and the runtime controls: teleports,
kinematic targets, type changes, enabling, motion locks, sleep controls,
forced sleep or wake and the fast-rotation switch (body.h:64-121;
body.c:170-330, 387-404, 531-823, 910-958) on the host.  With valid and
refused arguments they leave the world with the reference's hash, getters
and journal bytes, the reference's journal of them replays here to the
same world, and hostile records are refused whole (world.c:2323-2465,
2904-2928).  Stepping after these commands is covered on the device by
test_body_commands_gpu.py."""
import ctypes as C
import struct

from maul3d_b200 import abi
from maul3d_b200.abi import SCENE_TOWERS, SCENE_UNEVEN

V = abi.m3Vec3
P = abi.m3Pos3
Q = abi.m3Quat


def _commands(lib, wid):
    w0 = wid.index1 - 1
    for k in range(5):
        b = abi.m3BodyId(3 + k, w0, 0)
        lib.m3Body_ApplyForceAtPoint(b, V(2.0 * k, 0.5, -1.0), P(0.25 * k, 3.0, -0.5))
        lib.m3Body_ApplyLinearImpulseAtPoint(b, V(0.5, -1.5, 0.25 * k), P(1.0, 0.5 * k, 2.0))
        lib.m3Body_SetMotionLocks(b, [0x01, 0x12, 0x3F, 0x24, 0x00][k])
        lib.m3Body_SetAllowFastRotation(b, k % 2 == 0)
    b = abi.m3BodyId(4, w0, 0)
    lib.m3Body_ApplyForceAtPoint(b, V(float("nan"), 0.0, 0.0), P(0.0, 0.0, 0.0))   # refused
    lib.m3Body_ApplyLinearImpulseAtPoint(b, V(1.0, 0.0, 0.0), P(float("inf"), 0.0, 0.0))
    lib.m3Body_SetMotionLocks(b, 0x40)                                             # refused
    lib.m3Body_SetMotionLocks(b, 0x108)                                            # refused
    static = abi.m3BodyId(1, w0, 0)
    lib.m3Body_ApplyForceAtPoint(static, V(1.0, 1.0, 1.0), P(0.0, 1.0, 0.0))      # not dynamic
    lib.m3Body_ApplyLinearImpulseAtPoint(static, V(1.0, 1.0, 1.0), P(0.0, 1.0, 0.0))
    lib.m3Body_SetMotionLocks(static, 0x07)
    lib.m3Body_SetAllowFastRotation(abi.m3BodyId(6, w0, 0), True)
    lib.m3Body_SetAllowFastRotation(abi.m3BodyId(6, w0, 0), False)
    stale = abi.m3BodyId(3, w0, 9)
    lib.m3Body_SetMotionLocks(stale, 0x01)
    lib.m3Body_ApplyForceAtPoint(stale, V(1.0, 0.0, 0.0), P(0.0, 0.0, 0.0))
    _controls(lib, wid)


def _controls(lib, wid):
    w0 = wid.index1 - 1
    b = [abi.m3BodyId(k, w0, 0) for k in range(12)]
    half = 0.5 ** 0.5
    lib.m3Body_SetAwake(b[8], False)
    lib.m3Body_SetAwake(b[9], False)
    lib.m3Body_SetTransform(b[8], P(4.0, 6.0, -2.0), Q(0.0, half, 0.0, half))
    lib.m3Body_SetTransform(b[9], P(1.0, 2.0, 3.0), Q(0.0, 0.0, 0.0, 2.0))      # refused
    lib.m3Body_SetTransform(b[9], P(float("nan"), 2.0, 3.0), Q(0.0, 0.0, 0.0, 1.0))
    lib.m3Body_SetTargetTransform(b[9], P(1.0, 2.0, 3.0), Q(0.0, 0.0, 0.0, 1.0))  # not kinematic
    lib.m3Body_SetType(b[10], 1)
    lib.m3Body_SetTargetTransform(b[10], P(0.5, 3.0, 0.5), Q(0.0, 0.0, half, half))
    lib.m3Body_SetType(b[11], 0)
    lib.m3Body_SetType(b[11], 2)
    lib.m3Body_SetType(b[7], 2)                                                   # same type
    lib.m3Body_SetType(b[6], 5)                                                   # refused
    lib.m3Body_SetEnabled(b[5], False)
    lib.m3Body_SetEnabled(b[4], False)
    lib.m3Body_SetEnabled(b[4], True)
    lib.m3Body_SetSleepControls(b[3], 0.2, False)
    lib.m3Body_SetSleepControls(b[2], 0.0, True)
    lib.m3Body_SetSleepControls(b[2], -1.0, True)                                 # refused
    lib.m3Body_SetSleepControls(b[2], float("inf"), True)                         # refused
    lib.m3Body_SetAwake(b[1], False)                                              # static
    lib.m3Body_SetAwake(b[9], True)
    lib.m3Body_SetName(b[3], b"crate")
    lib.m3Body_SetName(b[4], b"a name longer than thirty-one bytes is cut")
    lib.m3Body_SetName(b[5], None)
    lib.m3Body_SetName(b[3], b"")
    lib.m3Body_SetName(b[6], b"lantern")


def _engines(m3, oracle):
    g = abi.bind_snapshot(abi.bind_body_commands(m3.lib))
    r = abi.bind_snapshot(abi.bind_body_commands(oracle.lib()))
    return g, r


def _journal(lib, wid, action):
    buf = (C.c_uint8 * 8192)()
    assert lib.m3World_JournalBegin(wid, buf, 8192)
    action()
    n = lib.m3World_JournalEnd(wid)
    assert n >= 0
    return bytes(buf[:n])


def _without_world_index(journal: bytes) -> bytes:
    """The records with the world0 half of every body id cleared (replay
    retargets it to the replaying world)."""
    out = bytearray(journal)
    cursor = 0
    while cursor < len(out):
        op, n = struct.unpack_from("<ii", out, cursor)
        out[cursor + 12:cursor + 14] = b"\0\0"
        cursor += 8 + n
    return bytes(out)


def _snapshot(lib, wid):
    n = lib.m3World_SnapshotSize(wid)
    buf = (C.c_uint8 * n)()
    assert lib.m3World_Snapshot(wid, buf, n) == n
    return bytes(buf)


def _getters(lib, wid, count):
    w0 = wid.index1 - 1
    rows = []
    for i in range(1, count + 1):
        b = abi.m3BodyId(i, w0, 0)
        rows.append((lib.m3Body_GetMotionLocks(b), lib.m3Body_GetAllowFastRotation(b),
                     lib.m3Body_GetType(b), lib.m3Body_GetUserData(b), lib.m3Body_IsEnabled(b),
                     lib.m3Body_IsAwake(b), lib.m3Body_GetName(b)))
    stale = abi.m3BodyId(2, w0, 7)
    rows.append((lib.m3Body_GetMotionLocks(stale), lib.m3Body_GetAllowFastRotation(stale),
                 lib.m3Body_GetType(stale), lib.m3Body_GetUserData(stale),
                 lib.m3Body_IsEnabled(stale), lib.m3Body_IsAwake(stale),
                 lib.m3Body_GetName(stale)))
    return rows


def test_body_commands_match_the_reference(m3, oracle):
    glib, rlib = _engines(m3, oracle)
    for scene, seed, param in ((SCENE_UNEVEN, 31, 40), (SCENE_TOWERS, 32, 2)):
        g = m3.World.scene(scene, seed, param)
        r = oracle.RefWorld.scene(scene, seed, param)
        gj = _journal(glib, g.id, lambda: _commands(glib, g.id))
        rj = _journal(rlib, r.id, lambda: _commands(rlib, r.id))
        assert _without_world_index(gj) == _without_world_index(rj) and len(rj) > 0
        assert g.hash() == r.hash()
        assert _getters(glib, g.id, 12) == _getters(rlib, r.id, 12)
        w0 = g.id.index1 - 1
        assert glib.m3Body_GetMotionLocks(abi.m3BodyId(5, w0, 0)) == 0x3F
        assert glib.m3Body_GetAllowFastRotation(abi.m3BodyId(5, w0, 0))
        assert glib.m3Body_GetName(abi.m3BodyId(4, w0, 0)) == b"a name longer than thirty-one b"
        assert glib.m3Body_GetName(abi.m3BodyId(6, w0, 0)) == b"lantern"
        # Names, locks and the other controls are in the snapshot bytes.
        assert _snapshot(glib, g.id) == _snapshot(rlib, r.id)
        g.destroy()
        r.destroy()


def test_reference_journal_of_body_commands_replays_here(m3, oracle):
    glib, rlib = _engines(m3, oracle)
    r = oracle.RefWorld.scene(SCENE_UNEVEN, 33, 40)
    journal = _journal(rlib, r.id, lambda: _commands(rlib, r.id))
    g = m3.World.scene(SCENE_UNEVEN, 33, 40)
    buf = (C.c_uint8 * len(journal)).from_buffer_copy(journal)
    assert glib.m3World_JournalReplay(g.id, buf, len(journal))
    assert g.hash() == r.hash()
    assert _snapshot(glib, g.id) == _snapshot(rlib, r.id)
    # A restore brings the names back.
    g2 = m3.World.scene(SCENE_UNEVEN, 33, 40)
    snap = _snapshot(rlib, r.id)
    sbuf = (C.c_uint8 * len(snap)).from_buffer_copy(snap)
    assert glib.m3World_Restore(g2.id, sbuf, len(snap))
    assert glib.m3Body_GetName(abi.m3BodyId(6, g2.id.index1 - 1, 0)) == b"lantern"
    assert _snapshot(glib, g2.id) == snap
    g2.destroy()
    r.destroy()
    g.destroy()


def test_name_records_keep_bytes_up_to_the_terminator(m3, oracle):
    # The reference forces the last byte to zero and copies up to the
    # first zero: bytes after it never reach the world.
    glib, rlib = _engines(m3, oracle)
    g = m3.World.scene(SCENE_UNEVEN, 35, 40)
    r = oracle.RefWorld.scene(SCENE_UNEVEN, 35, 40)
    for wid, lib in ((g.id, glib), (r.id, rlib)):
        body = bytes(abi.m3BodyId(3, wid.index1 - 1, 0))
        rec = abi.journal_record(68, body + b"ab\0junk" + b"z" * 25)
        buf = (C.c_uint8 * len(rec)).from_buffer_copy(rec)
        assert lib.m3World_JournalReplay(wid, buf, len(rec))
        assert lib.m3Body_GetName(abi.m3BodyId(3, wid.index1 - 1, 0)) == b"ab"
        short = abi.journal_record(68, body + b"ab")
        buf = (C.c_uint8 * len(short)).from_buffer_copy(short)
        assert not lib.m3World_JournalReplay(wid, buf, len(short))
    assert _snapshot(glib, g.id) == _snapshot(rlib, r.id)
    g.destroy()
    r.destroy()


def test_hostile_body_records_are_refused_whole(m3, oracle):
    glib, rlib = _engines(m3, oracle)
    g = m3.World.scene(SCENE_UNEVEN, 34, 40)
    r = oracle.RefWorld.scene(SCENE_UNEVEN, 34, 40)
    before = g.hash()
    w0 = g.id.index1 - 1
    body = bytes(abi.m3BodyId(3, w0, 0))
    stale = bytes(abi.m3BodyId(3, w0, 5))
    v = C.string_at(C.byref(V(1.0, 0.0, 0.0)), 12)
    p = C.string_at(C.byref(P(0.0, 1.0, 0.0)), 24)
    good = abi.journal_record(36, body + struct.pack("<I", 0x01))
    for bad in (abi.journal_record(30, body + C.string_at(C.byref(V(float("nan"), 0.0, 0.0)), 12)
                                   + bytes(4) + p),
                abi.journal_record(31, body + v + bytes(4) + C.string_at(
                    C.byref(P(0.0, float("inf"), 0.0)), 24)),
                abi.journal_record(31, body + v + bytes(4) + p[:20]),
                abi.journal_record(30, stale + v + bytes(4) + p),
                abi.journal_record(65, body + struct.pack("<I", 2)),
                abi.journal_record(36, stale + struct.pack("<I", 1)),
                abi.journal_record(36, body + struct.pack("<H", 1)),
                abi.journal_record(32, body + C.string_at(C.byref(P(0.0, 1.0, 0.0)), 24) +
                                   struct.pack("<4f", 0.0, 0.0, 0.0, 1.5)),
                abi.journal_record(33, stale + C.string_at(C.byref(P(0.0, 1.0, 0.0)), 24) +
                                   struct.pack("<4f", 0.0, 0.0, 0.0, 1.0)),
                abi.journal_record(32, body + struct.pack("<3d", 0.0, float("nan"), 0.0) +
                                   struct.pack("<4f", 0.0, 0.0, 0.0, 1.0)),
                abi.journal_record(35, stale + struct.pack("<i", 1)),
                abi.journal_record(38, body + struct.pack("<i", 1)[:3]),
                abi.journal_record(37, body + struct.pack("<fi", 0.5, 1)[:4])):
        stream = good + bad
        gbuf = (C.c_uint8 * len(stream)).from_buffer_copy(stream)
        assert not glib.m3World_JournalReplay(g.id, gbuf, len(stream))
        assert g.hash() == before
        # The reference refuses the same streams.
        rbuf = (C.c_uint8 * len(stream)).from_buffer_copy(stream)
        assert not rlib.m3World_JournalReplay(r.id, rbuf, len(stream))
    # Lock records carry a uint32; the reference keeps the low six bits.
    wide = abi.journal_record(36, body + struct.pack("<I", 0x1C2))
    gbuf = (C.c_uint8 * len(wide)).from_buffer_copy(wide)
    rbuf = (C.c_uint8 * len(wide)).from_buffer_copy(wide)
    r2 = oracle.RefWorld.scene(SCENE_UNEVEN, 34, 40)
    assert glib.m3World_JournalReplay(g.id, gbuf, len(wide))
    assert rlib.m3World_JournalReplay(r2.id, rbuf, len(wide))
    assert g.hash() == r2.hash()
    assert glib.m3Body_GetMotionLocks(abi.m3BodyId(3, w0, 0)) == 0x02
    # A type record keeps its low byte in both; one that names no body type
    # is refused here (the reference would store a type no path knows).
    for value, ok in ((0x102, True), (7, False)):
        rec = abi.journal_record(34, body + struct.pack("<i", value))
        gbuf = (C.c_uint8 * len(rec)).from_buffer_copy(rec)
        rbuf = (C.c_uint8 * len(rec)).from_buffer_copy(rec)
        assert bool(glib.m3World_JournalReplay(g.id, gbuf, len(rec))) == ok
        if ok:
            assert rlib.m3World_JournalReplay(r2.id, rbuf, len(rec))
            assert g.hash() == r2.hash()
    g.destroy()
    r.destroy()
    r2.destroy()


def test_mixed_host_journals_replay_both_ways(m3, oracle):
    # Body, shape and joint commands and world settings recorded here
    # replay in the reference, and the reference's in this library: both
    # worlds end with the same hash and snapshot bytes.
    import test_joint_commands as joints
    import test_shape_commands as shapes
    import test_world_settings as settings

    def bind(lib):
        for f in (abi.bind_body_commands, abi.bind_shape_commands, abi.bind_joint_commands,
                  abi.bind_settings, abi.bind_snapshot):
            lib = f(lib)
        return lib

    glib, rlib = bind(m3.lib), bind(oracle.lib())

    def session(lib, wid):
        _commands(lib, wid)
        shapes._commands(lib, wid)
        joints._commands(lib, wid)
        settings._apply_settings(lib, wid)

    g = m3.World.scene(SCENE_UNEVEN, 36, 60)
    r = oracle.RefWorld.scene(SCENE_UNEVEN, 36, 60)
    gj = _journal(glib, g.id, lambda: session(glib, g.id))
    rj = _journal(rlib, r.id, lambda: session(rlib, r.id))
    assert _without_world_index(gj) == _without_world_index(rj)
    g2 = m3.World.scene(SCENE_UNEVEN, 36, 60)
    r2 = oracle.RefWorld.scene(SCENE_UNEVEN, 36, 60)
    gbuf = (C.c_uint8 * len(rj)).from_buffer_copy(rj)
    rbuf = (C.c_uint8 * len(gj)).from_buffer_copy(gj)
    assert glib.m3World_JournalReplay(g2.id, gbuf, len(rj))
    assert rlib.m3World_JournalReplay(r2.id, rbuf, len(gj))
    assert g.hash() == r.hash() == g2.hash() == r2.hash()
    assert _snapshot(glib, g2.id) == _snapshot(rlib, r2.id) == _snapshot(rlib, r.id)
    for w in (g, r, g2, r2):
        w.destroy()
