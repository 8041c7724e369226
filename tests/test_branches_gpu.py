"""Solver branches no other scene reaches (needs a B200).

* The overflow colour (solver.c:2750-2810, BuildColoring; :2845-2877,
  RunColored): a plank carrying more constraints than there are graph
  colours puts the surplus in colour 16, which runs serially.  The
  device's colour count of every step (m3World_GetCounters().colorCount,
  17 when the overflow colour is used) must equal the reference's, and
  the world hash must match after every step.
* Restitution (solver.c:2879-2906): bodies with restitution 0.3-0.8
  dropped on a bouncy ground and on each other; hash parity every step,
  and the bodies really bounce.
"""
import numpy as np
import pytest

from conftest import cuda_available
from maul3d_b200.abi import SCENE_BOUNCE, SCENE_PLANK

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

DT = 1.0 / 60.0


@pytest.mark.parametrize("seed,boxes", [(1, 25), (2, 36)])
def test_overflow_colour_matches_the_reference_every_step(m3, oracle, seed, boxes):
    g = m3.World.scene(SCENE_PLANK, seed, boxes)
    r = oracle.RefWorld.scene(SCENE_PLANK, seed, boxes)
    assert g.hash() == r.hash()
    overflow_steps = 0
    for s in range(90):
        g.step(DT, 4, 1)
        r.step(DT, 4, 1)
        assert g.hash() == r.hash(), f"step {s + 1}"
        want = int(oracle.lib().m3o_last_color_count(r.id))
        got = m3.counters(g)["colorCount"]
        assert got == want, f"step {s + 1}: {got} colours on the device, {want} in the reference"
        overflow_steps += int(got == 17)
    assert overflow_steps >= 30, "the scene no longer reaches the overflow colour"
    g.destroy()
    r.destroy()


@pytest.mark.parametrize("seed,count", [(3, 40), (4, 90)])
def test_restitution_matches_the_reference_every_step(m3, oracle, seed, count):
    g = m3.World.scene(SCENE_BOUNCE, seed, count)
    r = oracle.RefWorld.scene(SCENE_BOUNCE, seed, count)
    assert g.hash() == r.hash()
    rebounds = 0
    for s in range(150):
        g.step(DT, 4, 1)
        r.step(DT, 4, 1)
        assert g.hash() == r.hash(), f"step {s + 1}"
        if s % 10 == 9:
            rebounds += int(np.sum(g.state().lin[:, 1] > 1.0))
    assert rebounds > 0, "nothing bounced: the restitution pass was not exercised"
    g.destroy()
    r.destroy()
