"""Distinct worlds stepped from distinct host threads (needs a B200).

The reference promises that distinct worlds may be stepped on distinct
threads at once, each with the result it gets alone (include/maul3d/
world.h:183-195, test/test_concurrency.c).  Here three host threads each
drive their own world through the drop-in m3World_Step (ctypes releases
the interpreter lock for the call), one of them also snapshotting its
world between steps; every world's hash after every step must equal the
reference engine's for the same world.
"""
import ctypes as C
import threading

import pytest

from conftest import cuda_available
from maul3d_b200.abi import SCENE_SHOTS, SCENE_TERRAIN, SCENE_UNEVEN

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

STEPS = 40


def test_three_threads_step_three_worlds_like_the_reference(m3, oracle):
    specs = [(SCENE_UNEVEN, 61, 300), (SCENE_TERRAIN, 62, 80), (SCENE_SHOTS, 63, 20)]
    want = []
    for spec in specs:
        r = oracle.RefWorld.scene(*spec)
        want.append([int(h) for h in r.trace(1.0 / 60.0, 4, STEPS)])
        r.destroy()
    worlds = [m3.World.scene(*spec) for spec in specs]
    got = [[] for _ in specs]
    errors = []
    start = threading.Barrier(len(specs))

    def drive(k):
        try:
            start.wait()
            for _ in range(STEPS):
                m3.lib.m3World_Step(worlds[k].id, C.c_float(1.0 / 60.0), 4)
                code = m3.lib.m3gpu_last_error()
                if code != m3.M3GPU_OK:
                    errors.append((k, code, m3.lib.m3gpu_last_error_message().decode()))
                    return
                got[k].append(int(m3.lib.m3World_Hash(worlds[k].id)))
                if k == 2:
                    # A reader on the same thread between its steps.
                    m3.snapshot(worlds[k])
        except Exception as exc:  # noqa: BLE001 - reported below
            errors.append((k, repr(exc)))

    threads = [threading.Thread(target=drive, args=(k,)) for k in range(len(specs))]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=600)
    assert not any(t.is_alive() for t in threads), "a stepping thread did not finish"
    assert not errors, errors
    for k in range(len(specs)):
        assert got[k] == want[k], f"world {k}: first mismatch at step " \
            f"{next(i for i in range(STEPS) if got[k][i] != want[k][i]) + 1}"
    for w in worlds:
        w.destroy()
