"""Shape materials and flags (shape.h:271-303; shape.c:1351-1363,
1387-1410, 1463-1600) on the host: friction, restitution, rolling
resistance, density (with and without the body's mass rebuilt) and the
hit-event and pre-solve flags, with valid and refused values, leave the
world with the reference's hash, getters and journal bytes; the
reference's journal of them replays here to the same world, and hostile
records are refused whole as the reference's replay refuses them
(world.c:2500-2555, 3021-3049)."""
import ctypes as C
import struct

from maul3d_b200 import abi
from maul3d_b200.abi import SCENE_TOWERS, SCENE_UNEVEN


def _commands(lib, wid):
    w0 = wid.index1 - 1
    s = [abi.m3ShapeId(k, w0, 0) for k in range(14)]
    for k in range(2, 8):
        lib.m3Shape_SetFriction(s[k], 0.1 * k)
        lib.m3Shape_SetRestitution(s[k], 0.05 * k)
        lib.m3Shape_SetRollingResistance(s[k], 0.02 * k)
        lib.m3Shape_EnableHitEvents(s[k], k % 2 == 0)
        lib.m3Shape_EnablePreSolve(s[k], k % 3 == 0)
    lib.m3Shape_SetDensity(s[8], 2.5, True)
    lib.m3Shape_SetDensity(s[9], 0.5, False)
    lib.m3Shape_SetDensity(s[1], 3.0, True)                      # a static body's shape
    lib.m3Shape_SetFriction(s[10], -0.5)                         # refused
    lib.m3Shape_SetRestitution(s[10], float("nan"))              # refused
    lib.m3Shape_SetRollingResistance(s[10], float("inf"))        # refused
    lib.m3Shape_SetDensity(s[10], 0.0, True)                     # refused
    lib.m3Shape_SetDensity(s[10], -1.0, True)                    # refused
    stale = abi.m3ShapeId(3, w0, 9)
    lib.m3Shape_SetFriction(stale, 0.5)
    lib.m3Shape_EnableHitEvents(stale, True)


def _getters(lib, wid):
    w0 = wid.index1 - 1
    rows = []
    for k in list(range(1, 14)) + [-3]:
        s = abi.m3ShapeId(abs(k), w0, 0 if k > 0 else 9)
        b = lib.m3Shape_GetBody(s)
        rows.append((lib.m3Shape_GetFriction(s), lib.m3Shape_GetRestitution(s),
                     lib.m3Shape_GetRollingResistance(s), lib.m3Shape_GetDensity(s),
                     lib.m3Shape_AreHitEventsEnabled(s), lib.m3Shape_IsPreSolveEnabled(s),
                     (b.index1, b.generation)))
    return rows


def _engines(m3, oracle):
    g = abi.bind_snapshot(abi.bind_shape_commands(m3.lib))
    r = abi.bind_snapshot(abi.bind_shape_commands(oracle.lib()))
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


def test_shape_commands_match_the_reference(m3, oracle):
    glib, rlib = _engines(m3, oracle)
    for scene, seed, param in ((SCENE_UNEVEN, 41, 40), (SCENE_TOWERS, 42, 2)):
        g = m3.World.scene(scene, seed, param)
        r = oracle.RefWorld.scene(scene, seed, param)
        gj = _journal(glib, g.id, lambda: _commands(glib, g.id))
        rj = _journal(rlib, r.id, lambda: _commands(rlib, r.id))
        assert _without_world_index(gj) == _without_world_index(rj) and len(rj) > 0
        assert g.hash() == r.hash()
        assert _getters(glib, g.id) == _getters(rlib, r.id)
        g.destroy()
        r.destroy()


def test_reference_journal_of_shape_commands_replays_here(m3, oracle):
    glib, rlib = _engines(m3, oracle)
    r = oracle.RefWorld.scene(SCENE_UNEVEN, 43, 40)
    journal = _journal(rlib, r.id, lambda: _commands(rlib, r.id))
    g = m3.World.scene(SCENE_UNEVEN, 43, 40)
    buf = (C.c_uint8 * len(journal)).from_buffer_copy(journal)
    assert glib.m3World_JournalReplay(g.id, buf, len(journal))
    assert g.hash() == r.hash()
    assert _getters(glib, g.id) == _getters(rlib, r.id)
    r.destroy()
    g.destroy()


def test_hostile_shape_records_are_refused_whole(m3, oracle):
    glib, rlib = _engines(m3, oracle)
    g = m3.World.scene(SCENE_UNEVEN, 44, 40)
    r = oracle.RefWorld.scene(SCENE_UNEVEN, 44, 40)
    before = g.hash()
    w0 = g.id.index1 - 1
    shape = bytes(abi.m3ShapeId(3, w0, 0))
    stale = bytes(abi.m3ShapeId(3, w0, 5))
    good = abi.journal_record(40, shape + struct.pack("<f", 0.25))
    for bad in (abi.journal_record(40, shape + struct.pack("<f", -0.25)),
                abi.journal_record(41, shape + struct.pack("<f", float("nan"))),
                abi.journal_record(42, stale + struct.pack("<f", 0.5)),
                abi.journal_record(43, shape + struct.pack("<fi", 0.0, 1)),
                abi.journal_record(43, shape + struct.pack("<f", 1.0)),
                abi.journal_record(50, stale + struct.pack("<i", 1)),
                abi.journal_record(51, shape + struct.pack("<h", 1))):
        stream = good + bad
        gbuf = (C.c_uint8 * len(stream)).from_buffer_copy(stream)
        assert not glib.m3World_JournalReplay(g.id, gbuf, len(stream))
        assert g.hash() == before
        rbuf = (C.c_uint8 * len(stream)).from_buffer_copy(stream)
        assert not rlib.m3World_JournalReplay(r.id, rbuf, len(stream))
    g.destroy()
    r.destroy()
