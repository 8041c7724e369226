"""Wide worlds: one world's substep loop over the whole grid (needs a B200).

A single large world runs its substep loop as a cooperative grid of many
blocks, the levels of its joint/contact schedule separated by grid
barriers (the reference fans one world's same-colour batches out to host
threads, solver.c:2845-2877).  The result must not depend on it: every
scene here is stepped on the wide path and its world hash compared with
the reference engine's after every step.  Small scenes are forced onto
the wide path (m3gpu_set_wide_min_shapes) so that the overflow colour,
restitution, revolute chains and breaking fixed joints all run on it.
"""
import pytest

from conftest import cuda_available
from maul3d_b200.abi import (SCENE_BOUNCE, SCENE_CITY, SCENE_PLANK, SCENE_TOWERS,
                             SCENE_UNEVEN)

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

DT = 1.0 / 60.0


@pytest.fixture
def wide_everywhere(m3):
    previous = m3.set_wide_min_shapes(1)
    yield
    m3.set_wide_min_shapes(previous)


@pytest.mark.parametrize("scene,seed,param,substeps,steps", [
    (SCENE_PLANK, 5, 30, 4, 60),
    (SCENE_BOUNCE, 6, 60, 4, 90),
    (SCENE_UNEVEN, 7, 400, 4, 60),
    (SCENE_TOWERS, 8, 6, 4, 90),
    (SCENE_CITY, 9, 3, 8, 45),
])
def test_forced_wide_path_matches_the_reference(m3, oracle, wide_everywhere, scene, seed,
                                                 param, substeps, steps):
    g = m3.World.scene(scene, seed, param)
    r = oracle.RefWorld.scene(scene, seed, param)
    assert g.hash() == r.hash()
    for s in range(steps):
        g.step(DT, substeps, 1)
        r.step(DT, substeps, 1)
        if g.hash() != r.hash():
            pytest.fail(f"step {s + 1}: {g.state().first_difference(r.state())}")
    g.destroy()
    r.destroy()


def test_city_world_goes_wide_and_matches_the_reference(m3, oracle):
    """30 towers (6,121 bodies, 13,800 breakable fixed joints, 120
    projectiles): above the default threshold, so wide by default."""
    g = m3.World.scene(SCENE_CITY, 5, 30)
    r = oracle.RefWorld.scene(SCENE_CITY, 5, 30)
    assert g.hash() == r.hash()
    assert m3.counters(g)["shapeCount"] >= m3.set_wide_min_shapes(0)
    for s in range(30):
        g.step(DT, 8, 1)
        r.step(DT, 8, 1)
        assert g.hash() == r.hash(), f"step {s + 1}"
    g.destroy()
    r.destroy()
