"""Launch limits (GPU): a world whose substep shared-memory cache sits
just under 48 KB (the default per-block limit, which also has to hold the
kernels' static shared memory) steps as the first work of a fresh
process, with the reference's hash.  The dynamic shared-memory limit of
the kernels is raised explicitly for every launch that needs it, not
left to the default.
"""
import os
import subprocess
import sys

import pytest

from conftest import cuda_available
from maul3d_b200.abi import SCENE_MIXED

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# 557 bodies (558 body slots with the ground): 558 x (52 + 36) bytes of
# body cache and inverse inertia table = 49,120 bytes of dynamic shared
# memory for the 256-thread kernels.
SEED, BODIES, STEPS = 20261284, 557, 5

SCRIPT = f"""
import sys
sys.path.insert(0, {ROOT!r})
import maul3d_b200 as m3
m3.set_device(0)
w = m3.World.scene({SCENE_MIXED}, {SEED}, {BODIES})
m3.step_worlds([w], 1.0 / 60.0, 4, {STEPS})
print(w.hash())
"""


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")
def test_a_world_just_under_the_default_shared_memory_limit_steps_first(oracle):
    out = subprocess.run([sys.executable, "-c", SCRIPT], capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    r = oracle.RefWorld.scene(SCENE_MIXED, SEED, BODIES)
    r.step(1.0 / 60.0, 4, STEPS)
    assert int(out.stdout.strip().splitlines()[-1]) == r.hash()
    r.destroy()
