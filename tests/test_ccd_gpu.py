"""Continuous collision against static targets on the device (needs a
B200).

Small spheres, boxes and capsules shot at 25-60 m/s across a ring of
static boxes, spheres and capsules move more than half their thinnest
extent in a step, so the continuous phase sweeps them against the static
shapes whose tree leaves touch their swept boxes (solver.c:3081-3425):
the time of impact (distance.c:711-1215) pulls each back to its first
touch.  The world hash must equal the reference's after every step.
Odd seeds add a heightfield patch, which the reference sweeps as the
point at its origin.
"""
import pytest

from conftest import cuda_available
from maul3d_b200.abi import SCENE_SHOTS

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]


@pytest.mark.parametrize("seed,shots,steps", [(2, 12, 60), (3, 24, 60), (4, 48, 45), (5, 90, 40)])
def test_shots_every_step_matches_oracle(m3, oracle, seed, shots, steps):
    g = m3.World.scene(SCENE_SHOTS, seed, shots)
    r = oracle.RefWorld.scene(SCENE_SHOTS, seed, shots)
    assert g.hash() == r.hash()
    for s in range(steps):
        g.step(1.0 / 60.0, 4, 1)
        r.step(1.0 / 60.0, 4, 1)
        assert g.hash() == r.hash(), f"seed {seed}: step {s + 1}"


def test_shots_batch_equals_worlds_stepped_alone(m3, oracle):
    specs = [(SCENE_SHOTS, 21 + k, 10 + 6 * k) for k in range(6)]
    batch = [m3.World.scene(*s) for s in specs]
    m3.step_worlds(batch, 1.0 / 60.0, 4, 40)
    got = m3.hash_worlds(batch)
    for k, s in enumerate(specs):
        r = oracle.RefWorld.scene(*s)
        r.step(1.0 / 60.0, 4, 40)
        assert int(got[k]) == r.hash(), f"world {k} {s}"
