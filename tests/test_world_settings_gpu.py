"""World settings changed between device steps (needs a B200).

Worlds step on the device, then gravity, contact tuning, speed caps, the
restitution and hit thresholds, wind and the continuous and sleeping
switches change (sleeping turned off wakes the bodies that fell asleep)
and the worlds step on: every step's hash must equal the reference
engine's, which takes the same calls.
"""
import ctypes as C

import pytest

from conftest import cuda_available
from maul3d_b200 import abi
from maul3d_b200.abi import SCENE_BOUNCE, SCENE_SHOTS, SCENE_UNEVEN

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

DT = 1.0 / 60.0
V = abi.m3Vec3


def _retune(lib, wid):
    lib.m3World_SetGravity(wid, V(1.0, -6.0, 0.5))
    lib.m3World_SetContactTuning(wid, 40.0, 5.0, 2.0)
    lib.m3World_SetRestitutionThreshold(wid, 0.25)
    lib.m3World_SetMaximumLinearSpeed(wid, 50.0)
    lib.m3World_SetMaximumAngularSpeed(wid, 20.0)
    lib.m3World_SetHitEventThreshold(wid, 0.5)
    lib.m3World_SetWind(wid, V(0.0, 0.0, 1.0), 2.0, 1.5, 0.3)
    lib.m3World_EnableSleeping(wid, False)
    lib.m3World_EnableContinuous(wid, False)


@pytest.mark.parametrize("scene,seed,param", [(SCENE_UNEVEN, 81, 300), (SCENE_BOUNCE, 82, 50),
                                              (SCENE_SHOTS, 83, 20)])
def test_settings_between_device_steps_match_the_reference(m3, oracle, scene, seed, param):
    glib = abi.bind_settings(m3.lib)
    rlib = abi.bind_settings(oracle.lib())
    g = m3.World.scene(scene, seed, param)
    r = oracle.RefWorld.scene(scene, seed, param)
    for s in range(150):
        if s == 100:
            _retune(glib, g.id)
            _retune(rlib, r.id)
        if s == 130:
            glib.m3World_EnableSleeping(g.id, True)
            rlib.m3World_EnableSleeping(r.id, True)
            glib.m3World_EnableContinuous(g.id, True)
            rlib.m3World_EnableContinuous(r.id, True)
        g.step(DT, 4, 1)
        r.step(DT, 4, 1)
        assert g.hash() == r.hash(), f"step {s + 1}"
    g.destroy()
    r.destroy()
