"""Event streams and the packing autotuner on the host side (no device
calls): a world that has not stepped has empty streams, stale ids and a
missing count pointer behave like the reference's entries
(world.c:1472-1500: 0 and NULL), and the autotuner refuses invalid
arguments before any device work."""
import ctypes as C

from maul3d_b200 import abi
from maul3d_b200.abi import SCENE_BOUNCE


def test_unstepped_world_has_empty_streams(m3):
    lib = abi.bind_events(m3.lib)
    w = m3.World.scene(SCENE_BOUNCE, 3, 20)
    events = abi.read_events(lib, w.id)
    assert all((len(v) if isinstance(v, list) else v) == 0 for v in events.values())
    w.destroy()


def test_stale_world_and_null_count(m3):
    lib = abi.bind_events(m3.lib)
    w = m3.World.scene(SCENE_BOUNCE, 4, 20)
    stale = abi.m3WorldId(w.id.index1, w.id.generation)
    w.destroy()
    for name in abi.EVENT_STREAMS + ("m3World_JointBreakEvents", "m3World_BodyMoveEvents",
                                     "m3World_HitEvents"):
        n = C.c_int32(7)
        assert not getattr(lib, name)(stale, C.byref(n))
        assert n.value == 0
    assert lib.m3World_HitEventsDropped(stale) == 0
    live = m3.World.scene(SCENE_BOUNCE, 5, 20)
    fn = lib.m3World_ContactBeginEvents
    fn.argtypes = [abi.m3WorldId, C.c_void_p]
    assert not fn(live.id, None)
    fn.argtypes = [abi.m3WorldId, C.POINTER(C.c_int32)]
    live.destroy()


def test_autotuner_refuses_invalid_arguments(m3):
    w = m3.World.scene(SCENE_BOUNCE, 6, 20)
    ids = (abi.m3WorldId * 1)(w.id)
    best = abi.m3gpuPacking()
    ms = C.c_float(0.0)
    before = m3.get_packing()
    for dt, sub, steps in ((0.0, 4, 3), (1.0 / 60.0, 0, 3), (1.0 / 60.0, 4, -1)):
        rc = m3.lib.m3gpu_autotune_packing(ids, 1, dt, sub, steps, C.byref(best), C.byref(ms))
        assert rc == m3.M3GPU_ERR_INVALID
    assert m3.lib.m3gpu_autotune_packing(ids, 0, 1.0 / 60.0, 4, 3, None, None) != 0
    assert m3.get_packing() == before
    w.destroy()
