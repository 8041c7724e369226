"""Regenerate tests/golden/traces.json from the oracle (the reference
engine built from its own sources by oracle/Makefile).

Each case builds one seeded scene (maul3d_b200/csrc/scenes.c) in the
reference, steps it with the reference's m3World_Step and records the
reference's m3World_Hash after selected steps.  The GPU parity tests
compare the device path against these values on hosts where the
reference sources are absent.  Run from the repository root:

    python tests/golden/make_golden.py
"""
import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import ref  # noqa: E402

# (name, scene, seed, param, dt, substeps, steps, checkpoints)
CASES = [
    ("freefall8", 3, 0, 8, 1.0 / 60.0, 4, 60, [1, 2, 10, 60]),
    ("sphere_pyramid", 0, 0, 0, 1.0 / 60.0, 4, 300, [1, 10, 100, 300]),
    ("box_pyramid_4", 1, 0, 4, 1.0 / 60.0, 4, 200, [1, 50, 200]),
    ("box_pyramid_20", 1, 0, 20, 1.0 / 60.0, 4, 1000, [1, 10, 100, 300, 600, 1000]),
    ("uneven_32_s1", 2, 1, 32, 1.0 / 60.0, 4, 300, [1, 10, 100, 300]),
    ("uneven_200_s3", 2, 3, 200, 1.0 / 60.0, 4, 300, [1, 10, 100, 300]),
    ("uneven_600_s4", 2, 4, 600, 1.0 / 60.0, 4, 300, [1, 10, 100, 300]),
    ("uneven_2048_s5", 2, 5, 2048, 1.0 / 60.0, 4, 120, [1, 10, 60, 120]),
    ("towers_4_s7", 4, 7, 4, 1.0 / 60.0, 4, 240, [1, 10, 20, 60, 240]),
    ("towers_16_s8", 4, 8, 16, 1.0 / 60.0, 4, 180, [1, 15, 30, 90, 180]),
    ("terrain_30_s1", 5, 1, 30, 1.0 / 60.0, 4, 200, [1, 10, 50, 200]),
    ("terrain_60_s2", 5, 2, 60, 1.0 / 60.0, 4, 120, [1, 30, 120]),
    ("shots_24_s3", 6, 3, 24, 1.0 / 60.0, 4, 60, [1, 10, 30, 60]),
]


def main() -> None:
    out = {"generator": "tests/golden/make_golden.py", "cases": []}
    for name, scene, seed, param, dt, sub, steps, cps in CASES:
        w = ref.RefWorld.scene(scene, seed, param)
        h0 = w.hash()
        trace = w.trace(dt, sub, steps)
        assert w.scratch_overflow() == 0
        out["cases"].append({
            "name": name, "scene": scene, "seed": seed, "param": param, "dt": dt,
            "substeps": sub, "steps": steps, "hash0": f"{h0:016x}",
            "hashes": {str(c): f"{int(trace[c - 1]):016x}" for c in cps},
        })
        w.destroy()
        print(name, out["cases"][-1]["hashes"])
    path = Path(__file__).with_name("traces.json")
    path.write_text(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    main()
