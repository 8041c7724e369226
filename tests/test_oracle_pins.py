"""Pin the oracle before trusting it.

The oracle is the reference engine compiled from its own sources
(oracle/Makefile).  It must reproduce every golden value the reference
holds for this path: the seven scene hashes of bench/pins.txt (via the
reference's own bench/bench_main.c), the determinism gate of
test/test_determinism.c, and the committed trace fixtures generated
from it (tests/golden/make_golden.py).
"""
import subprocess

import pytest

from conftest import GOLDEN_CASES

# bench/pins.txt:1-7 of the reference.
BENCH_PINS = {
    "pyramid": "975f319f2f44cc5d",
    "hulljam": "7bb4425d3adc3a51",
    "meshfield": "8f1cff6668d2f3ec",
    "meshgrand": "26a920286c1e25e7",
    "voxfort": "6cefd9054a3e16f1",
    "cityblock": "0993058b33ad2d5e",
    "smoke10k": "bc84e0074315a0b3",
}


def test_oracle_reproduces_reference_bench_pins(oracle):
    if not oracle.BENCH_PATH.exists():
        pytest.skip("reference bench binary not built")
    hashes = oracle.run_bench(300)
    for scene, pin in BENCH_PINS.items():
        assert hashes.get(scene) == pin, f"{scene}: {hashes.get(scene)} != pinned {pin}"


def test_oracle_determinism_gate(oracle):
    if not oracle.DET_PATH.exists():
        pytest.skip("reference determinism test not built")
    out = subprocess.run([str(oracle.DET_PATH)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "M3_DET_HASH=500860239b0e26e7" in out.stdout
    assert "all four gates hold" in out.stdout


def test_oracle_sphere_pyramid_matches_bench_pin(oracle):
    # The product's scene generator builds the reference bench's
    # "pyramid" layout; the reference steps it to the pinned hash.
    w = oracle.RefWorld.scene(0)
    trace = w.trace(1.0 / 60.0, 4, 300)
    assert f"{int(trace[-1]):016x}" == BENCH_PINS["pyramid"]
    w.destroy()


@pytest.mark.parametrize("idx", range(GOLDEN_CASES))
def test_oracle_reproduces_golden_traces(oracle, golden, idx):
    case = golden["cases"][idx]
    w = oracle.RefWorld.scene(case["scene"], case["seed"], case["param"])
    assert f"{w.hash():016x}" == case["hash0"]
    trace = w.trace(case["dt"], case["substeps"], case["steps"])
    for step, h in case["hashes"].items():
        assert f"{int(trace[int(step) - 1]):016x}" == h, f"{case['name']} step {step}"
    assert w.scratch_overflow() == 0
    w.destroy()
