"""World settings (world.h:92-176, 288; world.c:785-1117) on the host:
every setter, with valid and refused values, leaves the world with the
reference's hash, getters and journal bytes, and the reference's journal
of those settings replays here to the same world (hostile records are
refused whole, the world untouched).  The stepping side is in
test_world_settings_gpu.py."""
import ctypes as C

from maul3d_b200 import abi
from maul3d_b200.abi import SCENE_BOUNCE, SCENE_UNEVEN

V = abi.m3Vec3


def _apply_settings(lib, wid):
    lib.m3World_SetGravity(wid, V(0.5, -7.5, 0.25))
    lib.m3World_SetGravity(wid, V(float("nan"), 0.0, 0.0))       # refused
    lib.m3World_SetContactTuning(wid, 45.0, 7.0, 2.5)
    lib.m3World_SetContactTuning(wid, 45.0, 0.0, 2.5)            # refused
    lib.m3World_SetRestitutionThreshold(wid, 0.5)
    lib.m3World_SetRestitutionThreshold(wid, -1.0)               # refused
    lib.m3World_SetMaximumLinearSpeed(wid, 120.0)
    lib.m3World_SetMaximumLinearSpeed(wid, 0.0)                  # refused
    lib.m3World_SetMaximumAngularSpeed(wid, 40.0)
    lib.m3World_SetHitEventThreshold(wid, 2.0)
    lib.m3World_EnableContinuous(wid, False)
    lib.m3World_EnableSleeping(wid, False)
    lib.m3World_EnableSleeping(wid, True)
    lib.m3World_SetWind(wid, V(0.0, 0.0, 2.0), 3.0, 0.5, 0.2)   # refused: not unit
    lib.m3World_SetWind(wid, V(0.6, 0.0, 0.8), 3.0, 0.5, 0.2)


def _engines(m3, oracle):
    g = abi.bind_snapshot(abi.bind_settings(m3.lib))
    r = abi.bind_snapshot(abi.bind_settings(oracle.lib()))
    return g, r


def _journal(lib, wid, action):
    buf = (C.c_uint8 * 4096)()
    assert lib.m3World_JournalBegin(wid, buf, 4096)
    action()
    n = lib.m3World_JournalEnd(wid)
    assert n >= 0
    return bytes(buf[:n])


def test_settings_match_the_reference(m3, oracle):
    glib, rlib = _engines(m3, oracle)
    for scene, seed, param in ((SCENE_BOUNCE, 21, 30), (SCENE_UNEVEN, 22, 100)):
        g = m3.World.scene(scene, seed, param)
        r = oracle.RefWorld.scene(scene, seed, param)
        gj = _journal(glib, g.id, lambda: _apply_settings(glib, g.id))
        rj = _journal(rlib, r.id, lambda: _apply_settings(rlib, r.id))
        assert gj == rj and len(rj) > 0
        assert g.hash() == r.hash()
        gg = glib.m3World_GetGravity(g.id)
        rg = rlib.m3World_GetGravity(r.id)
        assert (gg.x, gg.y, gg.z) == (rg.x, rg.y, rg.z) == (0.5, -7.5, 0.25)
        assert glib.m3World_IsSleepingEnabled(g.id) and rlib.m3World_IsSleepingEnabled(r.id)
        assert not glib.m3World_IsContinuousEnabled(g.id)
        assert not rlib.m3World_IsContinuousEnabled(r.id)
        g.destroy()
        r.destroy()


def test_reference_journal_of_settings_replays_here(m3, oracle):
    glib, rlib = _engines(m3, oracle)
    r = oracle.RefWorld.scene(SCENE_BOUNCE, 23, 30)
    journal = _journal(rlib, r.id, lambda: _apply_settings(rlib, r.id))
    g = m3.World.scene(SCENE_BOUNCE, 23, 30)
    buf = (C.c_uint8 * len(journal)).from_buffer_copy(journal)
    assert glib.m3World_JournalReplay(g.id, buf, len(journal))
    assert g.hash() == r.hash()
    r.destroy()
    g.destroy()


def test_hostile_setting_records_are_refused_whole(m3):
    glib = abi.bind_snapshot(abi.bind_settings(m3.lib))
    g = m3.World.scene(SCENE_BOUNCE, 24, 30)
    before = g.hash()
    good = abi.journal_record(39, C.string_at(C.byref(V(0.0, -5.0, 0.0)), 12))
    for bad in (abi.journal_record(39, C.string_at(C.byref(V(float("inf"), 0.0, 0.0)), 12)),
                abi.journal_record(44, bytes(C.c_float(1.0)) + bytes(C.c_float(-1.0)) +
                                   bytes(C.c_float(1.0))),
                abi.journal_record(66, bytes(C.c_float(0.0))),
                abi.journal_record(60, bytes(24)[:20])):
        stream = good + bad
        buf = (C.c_uint8 * len(stream)).from_buffer_copy(stream)
        assert not glib.m3World_JournalReplay(g.id, buf, len(stream))
        assert g.hash() == before
    g.destroy()
