"""Body commands at a world point and the runtime controls between device
steps (needs a B200).

Worlds step on the device; then forces and impulses at world points,
motion locks, the fast-rotation switch, teleports, forced sleep, a body
turned kinematic and servoed to a target, a body disabled and sleep
controls are applied (later some locks are lifted, the kinematic body
turns dynamic again and the disabled one comes back) and the worlds step
on: the locked components re-zero every substep (solver.c:4156-4177), the
switch bypasses the angular cap (solver.c:4131-4144), the target drives
the kinematic body's velocity.  Every step's hash must equal the
reference engine's, which takes the same calls.
"""
import pytest

from conftest import cuda_available
from maul3d_b200 import abi
from maul3d_b200.abi import SCENE_BOUNCE, SCENE_UNEVEN

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

DT = 1.0 / 60.0
V = abi.m3Vec3
P = abi.m3Pos3
Q = abi.m3Quat


def _command(lib, wid, lift):
    w0 = wid.index1 - 1
    for k in range(6):
        b = abi.m3BodyId(3 + 2 * k, w0, 0)
        if lift:
            lib.m3Body_SetMotionLocks(b, 0x00 if k % 2 else 0x08)
            continue
        lib.m3Body_ApplyLinearImpulseAtPoint(b, V(1.5, 4.0 + k, -0.5), P(0.5 * k, 2.0, 0.25))
        lib.m3Body_ApplyForceAtPoint(b, V(-3.0, 8.0, 2.0 * k), P(1.0, 0.5, -0.5 * k))
        lib.m3Body_SetMotionLocks(b, [0x01, 0x2A, 0x07, 0x38, 0x12, 0x3F][k])
        lib.m3Body_SetAllowFastRotation(b, k % 3 == 0)
    b = [abi.m3BodyId(k, w0, 0) for k in range(24)]
    half = 0.5 ** 0.5
    if lift:
        lib.m3Body_SetType(b[16], 2)
        lib.m3Body_SetEnabled(b[18], True)
        lib.m3Body_SetAwake(b[20], True)
        lib.m3Body_SetSleepControls(b[22], 0.0, True)
        return
    pos = lib.m3Body_GetPosition(b[14])
    lib.m3Body_SetTransform(b[14], P(pos.x + 0.5, pos.y + 3.0, pos.z), Q(0.0, half, 0.0, half))
    lib.m3Body_SetType(b[16], 1)
    pos = lib.m3Body_GetPosition(b[16])
    lib.m3Body_SetTargetTransform(b[16], P(pos.x, pos.y + 0.5, pos.z + 0.25),
                                  Q(0.0, 0.0, 0.258819, 0.9659258))
    lib.m3Body_SetEnabled(b[18], False)
    lib.m3Body_SetAwake(b[20], False)
    lib.m3Body_SetSleepControls(b[22], 0.3, False)
    lib.m3Body_SetSleepControls(b[23], 0.5, True)


@pytest.mark.parametrize("scene,seed,param", [(SCENE_UNEVEN, 91, 300), (SCENE_BOUNCE, 92, 50)])
def test_body_commands_between_device_steps_match_the_reference(m3, oracle, scene, seed, param):
    glib = abi.bind_body_commands(m3.lib)
    rlib = abi.bind_body_commands(oracle.lib())
    g = m3.World.scene(scene, seed, param)
    r = oracle.RefWorld.scene(scene, seed, param)
    for s in range(120):
        if s in (40, 80):
            _command(glib, g.id, s == 80)
            _command(rlib, r.id, s == 80)
        g.step(DT, 4, 1)
        r.step(DT, 4, 1)
        assert g.hash() == r.hash(), f"step {s + 1}"
    g.destroy()
    r.destroy()
