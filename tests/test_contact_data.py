"""Contact readback (body.h:99, shape.h:274; query.c:1330-1409) on the
host: a world restored from the reference's snapshot after it stepped
reads back the same contact entries, byte for byte, per body and per
shape, with truncation at the capacity and the reference's zero answers
for stale ids, a null buffer and a non-positive capacity."""
import ctypes as C

import pytest

from maul3d_b200 import abi
from maul3d_b200.abi import SCENE_BOX_PYRAMID, SCENE_TOWERS, SCENE_UNEVEN


def _read(fn, ident, capacity):
    buf = (abi.m3ContactData * max(capacity, 1))()
    n = fn(ident, buf, capacity)
    return n, bytes(buf)[:n * C.sizeof(abi.m3ContactData)]


def _snapshot(lib, wid):
    n = lib.m3World_SnapshotSize(wid)
    buf = (C.c_uint8 * n)()
    assert lib.m3World_Snapshot(wid, buf, n) == n
    return bytes(buf)


@pytest.mark.parametrize("scene,seed,param,steps", [(SCENE_UNEVEN, 61, 64, 60),
                                                    (SCENE_TOWERS, 62, 2, 30),
                                                    (SCENE_BOX_PYRAMID, 0, 6, 40)])
def test_contact_data_equals_the_references(m3, oracle, scene, seed, param, steps):
    glib = abi.bind_snapshot(abi.bind_contact_data(m3.lib))
    rlib = abi.bind_snapshot(abi.bind_contact_data(oracle.lib()))
    r = oracle.RefWorld.scene(scene, seed, param)
    r.step(1.0 / 60.0, 4, steps)
    snap = _snapshot(rlib, r.id)
    g = m3.World.scene(scene, seed, param)
    buf = (C.c_uint8 * len(snap)).from_buffer_copy(snap)
    assert glib.m3World_Restore(g.id, buf, len(snap))
    gw, rw = g.id.index1 - 1, r.id.index1 - 1
    seen = 0
    for k in range(1, 40):
        for cap in (16, 2):
            gn, gb = _read(glib.m3Body_GetContactData, abi.m3BodyId(k, gw, 0), cap)
            rn, rb = _read(rlib.m3Body_GetContactData, abi.m3BodyId(k, rw, 0), cap)
            assert gn == rn and _strip(gb, gw) == _strip(rb, rw), (k, cap)
            seen += gn
            gn, gb = _read(glib.m3Shape_GetContactData, abi.m3ShapeId(k, gw, 0), cap)
            rn, rb = _read(rlib.m3Shape_GetContactData, abi.m3ShapeId(k, rw, 0), cap)
            assert gn == rn and _strip(gb, gw) == _strip(rb, rw), (k, cap)
    assert seen > 0
    for lib, w0 in ((glib, gw), (rlib, rw)):
        assert _read(lib.m3Body_GetContactData, abi.m3BodyId(3, w0, 7), 8)[0] == 0
        assert _read(lib.m3Body_GetContactData, abi.m3BodyId(3, w0, 0), 0)[0] == 0
        assert lib.m3Body_GetContactData(abi.m3BodyId(3, w0, 0), None, 8) == 0
        assert _read(lib.m3Shape_GetContactData, abi.m3ShapeId(3, w0, 7), 8)[0] == 0
    g.destroy()
    r.destroy()


def _strip(raw: bytes, world0: int) -> bytes:
    """Entries with the world0 half of both shape ids cleared (each engine
    names its own world)."""
    out = bytearray(raw)
    size = C.sizeof(abi.m3ContactData)
    for base in range(0, len(out), size):
        for off in (4, 12):
            assert out[base + off:base + off + 2] == bytes(C.c_uint16(world0))
            out[base + off:base + off + 2] = b"\0\0"
    return bytes(out)
