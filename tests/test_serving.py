"""Serving (C4): replay containers in, final hashes out.

CPU: the M3J1 container codec (replay.c:15-136) encodes the reference's
bytes and refuses what it refuses.  GPU: a server fed containers of
reference snapshots and impulse journals answers each with the hash the
reference gives after m3World_Restore + m3World_JournalReplay, whatever
else shares the batch.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import cuda_available
from maul3d_b200 import abi
from maul3d_b200.abi import SCENE_MIXED, SCENE_TERRAIN, SCENE_TOWERS, SCENE_UNEVEN


def _snapshot(lib, wid) -> bytes:
    n = lib.m3World_SnapshotSize(wid)
    buf = (C.c_uint8 * n)()
    assert lib.m3World_Snapshot(wid, buf, n) == n
    return bytes(buf)


def _journal(rng, bodies: int, frames: int) -> bytes:
    """`frames` frames of 1-8 linear impulses of 1-50 N s on random bodies,
    each closed by a step of 1/60 s in 4 substeps."""
    out = b""
    for _ in range(frames):
        for _ in range(int(rng.integers(1, 9))):
            d = rng.normal(size=3)
            d = d / np.linalg.norm(d) * rng.uniform(1.0, 50.0)
            out += abi.journal_body_command(abi.OP_APPLY_LINEAR_IMPULSE,
                                            int(rng.integers(2, bodies + 1)), 0,
                                            [float(x) for x in d.astype(np.float32)])
        out += abi.journal_step(1.0 / 60.0, 4)
    return out


@pytest.fixture(scope="module")
def ref(oracle):
    return abi.bind_replay(abi.bind_snapshot(abi.bind_create(oracle.lib())))


def test_container_codec_matches_the_reference(m3, ref):
    rng = np.random.default_rng(3)
    snap = bytes(rng.integers(0, 256, 400, dtype=np.uint8))
    journal = _journal(rng, 50, 5)
    ours = abi.encode_container(m3.lib, snap, journal, 0x1234)
    theirs = abi.encode_container(ref, snap, journal, 0x1234)
    assert ours == theirs
    for lib in (m3.lib, ref):
        view = abi.m3ReplayView()
        buf = (C.c_uint8 * len(ours)).from_buffer_copy(ours)
        assert lib.m3ReplayDecode(buf, len(ours), C.byref(view))
        assert view.snapshotBytes == 400 and view.finalHash == 0x1234
        assert view.info.stepCount == 5
        bad = bytearray(ours)
        bad[16] ^= 1  # a header that lies about its step count
        buf = (C.c_uint8 * len(bad)).from_buffer_copy(bytes(bad))
        assert not lib.m3ReplayDecode(buf, len(bad), C.byref(view))
        info = abi.m3JournalInfo()
        j = (C.c_uint8 * len(journal)).from_buffer_copy(journal)
        assert lib.m3JournalDescribe(j, len(journal), C.byref(info))
        assert not lib.m3JournalDescribe(j, len(journal) - 1, C.byref(info))


def test_submit_refuses_a_bad_container(m3):
    server = m3.Server()
    with pytest.raises(m3.M3GpuError):
        server.submit(b"not a container at all, not even close....")
    server.close()


def _requests(oracle, ref, count, seed):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(count):
        if i % 5 == 4:
            scene, param = SCENE_TOWERS, 2
        elif i % 5 == 3:
            scene, param = SCENE_TERRAIN, int(rng.integers(40, 200))
        else:
            scene, param = SCENE_UNEVEN, int(rng.integers(200, 700))
        r = oracle.RefWorld.scene(scene, 900 + i, param)
        r.step(1.0 / 60.0, 4, int(rng.integers(1, 30)))
        snap = _snapshot(ref, r.id)
        journal = _journal(rng, r.body_count() - 1, int(rng.integers(4, 17)))
        jb = (C.c_uint8 * len(journal)).from_buffer_copy(journal)
        assert ref.m3World_JournalReplay(r.id, jb, len(journal))
        reqs.append((abi.encode_container(ref, snap, journal, r.hash()), r.hash()))
        r.destroy()
    return reqs


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")
def test_served_hashes_equal_restore_and_replay_on_the_reference(m3, oracle, ref):
    reqs = _requests(oracle, ref, 24, 7)
    server = m3.Server(max_active=10)
    tickets = [server.submit(c) for c, _ in reqs]
    done = server.run()
    server.close()
    for t, (_, expected) in zip(tickets, reqs):
        h, status = done[t]
        assert status == m3.M3GPU_OK
        assert h == expected, f"ticket {t}"


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")
def test_a_request_alone_and_in_a_crowd_gives_the_same_hash(m3, oracle, ref):
    reqs = _requests(oracle, ref, 6, 11)
    alone = m3.Server()
    t = alone.submit(reqs[0][0])
    h_alone = alone.run()[t][0]
    alone.close()
    crowd = m3.Server(max_active=3)
    ts = [crowd.submit(c) for c, _ in reqs]
    done = crowd.run()
    crowd.close()
    assert done[ts[0]][0] == h_alone == reqs[0][1]


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")
def test_unmodelled_content_completes_with_its_refusal(m3, oracle, ref):
    # A snapshot with a live water volume: restored nowhere, reported.
    from test_snapshot import _WaterVolumeDef, _WaterVolumeId
    lib = oracle.lib()
    lib.m3DefaultWaterVolumeDef.restype = _WaterVolumeDef
    lib.m3CreateWaterVolume.argtypes = [abi.m3WorldId, C.POINTER(_WaterVolumeDef)]
    lib.m3CreateWaterVolume.restype = _WaterVolumeId
    r = oracle.RefWorld.scene(SCENE_UNEVEN, 5, 64)
    wd = lib.m3DefaultWaterVolumeDef()
    wd.lo = abi.m3Pos3(-5.0, -1.0, -5.0)
    wd.hi = abi.m3Pos3(5.0, 0.5, 5.0)
    assert lib.m3CreateWaterVolume(r.id, C.byref(wd)).index1 > 0
    container = abi.encode_container(ref, _snapshot(ref, r.id), abi.journal_step(1 / 60, 4))
    good = _requests(oracle, ref, 1, 13)[0]
    server = m3.Server()
    bad_t = server.submit(container)
    good_t = server.submit(good[0])
    done = server.run()
    server.close()
    assert done[bad_t][1] == m3.M3GPU_ERR_UNSUPPORTED
    assert done[good_t] == (good[1], m3.M3GPU_OK)


def _mixed_requests(oracle, ref, count, seed, bodies=(200, 600)):
    """Containers of the served configuration's worlds (boxes, spheres and
    16-point hulls on a plane), each stepped a little on the reference,
    with the reference's hash after replaying the journal."""
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(count):
        r = oracle.RefWorld.scene(SCENE_MIXED, 500 + i, int(rng.integers(*bodies)))
        r.step(1.0 / 60.0, 4, int(rng.integers(1, 10)))
        snap = _snapshot(ref, r.id)
        journal = _journal(rng, r.body_count() - 1, int(rng.integers(4, 17)))
        jb = (C.c_uint8 * len(journal)).from_buffer_copy(journal)
        assert ref.m3World_JournalReplay(r.id, jb, len(journal))
        reqs.append((abi.encode_container(ref, snap, journal, r.hash()), r.hash()))
        r.destroy()
    return reqs


def test_a_stale_journal_is_refused_before_the_device(m3, oracle, ref):
    # Preparation (world, restore, journal) runs on the worker threads; a
    # journal naming a body the snapshot does not hold retires with
    # M3GPU_ERR_INVALID without the device being touched, on a machine
    # without one too.  Nothing stays held.
    r = oracle.RefWorld.scene(SCENE_MIXED, 3, 120)
    snap = _snapshot(ref, r.id)
    r.destroy()
    journal = (abi.journal_body_command(abi.OP_APPLY_LINEAR_IMPULSE, 100000, 0, [1.0, 0.0, 0.0]) +
               abi.journal_step(1 / 60, 4))
    container = abi.encode_container(ref, snap, journal)
    server = m3.Server()
    tickets = [server.submit(container) for _ in range(3)]
    done = server.run()
    stats = server.stats()
    server.close()
    assert all(done[t][1] == m3.M3GPU_ERR_INVALID for t in tickets)
    assert stats["refused"] == 3 and stats["completed"] == 0
    assert stats["heldBytes"] == 0 and stats["active"] == 0 and stats["preparing"] == 0


def test_preparation_starts_only_what_the_budget_holds(m3, oracle, ref):
    # Requests are counted against the device budget when their
    # preparation starts: with room for two and a half of them, at most
    # two are ever held (these are refused in preparation, so this runs
    # without a device).
    r = oracle.RefWorld.scene(SCENE_MIXED, 4, 300)
    snap = _snapshot(ref, r.id)
    r.destroy()
    journal = (abi.journal_body_command(abi.OP_APPLY_LINEAR_IMPULSE, 100000, 0, [1.0, 0.0, 0.0]) +
               abi.journal_step(1 / 60, 4))
    container = abi.encode_container(ref, snap, journal)
    one = m3.Server()
    one.submit(container)
    one.run()
    size = one.stats()["peakHeldBytes"]
    one.close()
    assert size > 0
    server = m3.Server(device_budget=int(2.5 * size))
    for _ in range(6):
        server.submit(container)
    server.run()
    stats = server.stats()
    server.close()
    assert stats["peakHeldBytes"] == 2 * size
    assert stats["refused"] == 6 and stats["heldBytes"] == 0


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")
def test_admission_keeps_within_the_device_budget(m3, oracle, ref):
    # Six requests of about the same size under a budget of two and a half
    # of them: never more than two held at once, every answer the
    # reference's, whatever the admission order did.
    reqs = _mixed_requests(oracle, ref, 6, 21, bodies=(300, 320))
    one = m3.Server()
    t = one.submit(reqs[0][0])
    assert one.run()[t] == (reqs[0][1], m3.M3GPU_OK)
    size = one.stats()["peakHeldBytes"]
    one.close()
    assert size > 0
    server = m3.Server(device_budget=int(2.5 * size))
    tickets = [server.submit(c) for c, _ in reqs]
    done = server.run()
    stats = server.stats()
    server.close()
    assert stats["peakHeldBytes"] <= int(2.5 * size)
    assert stats["peakActive"] <= 2
    assert stats["completed"] == len(reqs) and stats["heldBytes"] == 0
    for t, (_, expected) in zip(tickets, reqs):
        assert done[t] == (expected, m3.M3GPU_OK), f"ticket {t}"


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")
def test_served_hull_worlds_equal_the_reference(m3, oracle, ref):
    # The served configuration's worlds (16-point QuickHull hulls, boxes,
    # spheres) arriving while others run: submitted between ticks.
    reqs = _mixed_requests(oracle, ref, 12, 5)
    server = m3.Server(max_active=6)
    tickets, done = [], {}
    for k, (c, _) in enumerate(reqs):
        tickets.append(server.submit(c))
        if k % 3 == 2:
            server.tick()
            t, h, st = server.poll()
            done.update({int(t[i]): (int(h[i]), int(st[i])) for i in range(len(t))})
    done.update(server.run())
    server.close()
    for t, (_, expected) in zip(tickets, reqs):
        assert done[t] == (expected, m3.M3GPU_OK), f"ticket {t}"


def test_submissions_from_another_thread_are_all_answered(m3, oracle, ref):
    # A client thread submits while this thread ticks; every ticket comes
    # back once (refused in preparation here, so no device is needed).
    import threading
    r = oracle.RefWorld.scene(SCENE_MIXED, 6, 60)
    snap = _snapshot(ref, r.id)
    r.destroy()
    journal = (abi.journal_body_command(abi.OP_APPLY_LINEAR_IMPULSE, 100000, 0, [1.0, 0.0, 0.0]) +
               abi.journal_step(1 / 60, 4))
    container = abi.encode_container(ref, snap, journal)
    server = m3.Server()
    tickets = []
    client = threading.Thread(target=lambda: tickets.extend(server.submit(container)
                                                            for _ in range(40)))
    client.start()
    seen = {}
    while client.is_alive() or server.tick() > 0:
        server.tick()
        t, h, st = server.poll()
        for k in range(len(t)):
            assert int(t[k]) not in seen
            seen[int(t[k])] = int(st[k])
    client.join()
    server.tick()
    t, h, st = server.poll()
    seen.update({int(t[k]): int(st[k]) for k in range(len(t))})
    server.close()
    assert sorted(seen) == sorted(tickets) == list(range(1, 41))
    assert set(seen.values()) == {m3.M3GPU_ERR_INVALID}


def test_host_side_records_in_served_journals_are_refused(m3, oracle, ref):
    # World settings, shape materials and runtime controls change the
    # host image between frames: a served journal holding one completes
    # with the refusal.  The refusal comes while the request is prepared
    # on the host, before any device work.
    r = oracle.RefWorld.scene(SCENE_UNEVEN, 7, 64)
    snap = _snapshot(ref, r.id)
    w0 = r.id.index1 - 1
    records = (abi.journal_record(39, C.string_at(C.byref(abi.m3Vec3(0.0, -5.0, 0.0)), 12)),
               abi.journal_record(40, bytes(abi.m3ShapeId(3, w0, 0)) + bytes(C.c_float(0.5))),
               abi.journal_record(38, bytes(abi.m3BodyId(3, w0, 0)) + bytes(C.c_int32(0))),
               abi.journal_record(52, bytes(abi.m3JointId(2, w0, 0)) +
                                  bytes(C.c_int32(1)) + bytes(C.c_float(-0.5)) +
                                  bytes(C.c_float(0.5))))
    server = m3.Server()
    tickets = [server.submit(abi.encode_container(ref, snap, rec + abi.journal_step(1 / 60, 4)))
               for rec in records]
    done = server.run()
    server.close()
    for t in tickets:
        assert done[t] == (0, m3.M3GPU_ERR_UNSUPPORTED)
