"""The large single worlds at full size, step by step (needs a B200).

* The city: towers of 10 x 10 x 2 boxes welded by fixed joints that break
  at 500 N, with four projectiles per tower, 8 substeps -- the wide and
  overflow-prone colour paths, fixed-joint rows and joint breakage at
  scale.  300 towers (61,201 bodies, 138,000 joints) against the stock
  reference; 1000 towers (204,001 bodies, 460,000 joints), the large
  configuration itself, against the reference built with its step scratch
  cap raised (the stock build stalls on every step of it).
* The rain field at full size: 10,000 spheres, capsules and QuickHull
  hulls falling 5-100 m onto a 255 x 255 heightfield, all 600 steps (the
  heightfield narrowphase and the continuous phase at scale).

Each world is built by this library through the reference-named creation
API and stepped on the device (the wide path: one world over the whole
grid); its hash after every step must equal the reference's, recorded in
tests/golden/large_traces.json by tests/golden/make_large_golden.py.
"""
import json
from pathlib import Path

import pytest

from conftest import cuda_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

TRACES = Path(__file__).resolve().parent / "golden" / "large_traces.json"


def _cases():
    if not TRACES.exists():
        return []
    return [c["name"] for c in json.loads(TRACES.read_text())["cases"]]


@pytest.mark.parametrize("name", _cases())
def test_large_world_matches_the_reference_every_step(m3, name):
    case = next(c for c in json.loads(TRACES.read_text())["cases"] if c["name"] == name)
    g = m3.World.scene(case["scene"], case["seed"], case["param"])
    assert g.body_count() == case["bodies"]
    assert f"{g.hash():016x}" == case["hash0"]
    m3.reserve_worlds([g])
    m3.upload_worlds([g])
    for s, want in enumerate(case["trace"]):
        g.step(case["dt"], case["substeps"], 1)
        got = f"{int(m3.hash_worlds([g])[0]):016x}"
        assert got == want, f"{name}: step {s + 1} hash {got}, reference {want}"
    g.destroy()
