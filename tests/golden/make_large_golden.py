"""Regenerate tests/golden/large_traces.json: per-step world hashes of the
large single worlds, from the oracle (the reference engine built from its
own sources by oracle/Makefile).

Cases:
  city_300_s5    300 towers of 10 x 10 x 2 welded boxes and 1200 spheres
                 (61,201 bodies, 138,000 breakable fixed joints), the stock
                 reference build, 8 substeps, 30 steps.
  city_1000_s5   1000 towers (204,001 bodies, 460,000 joints): the stock
                 reference stalls on it (its 256 MB step scratch cap), so
                 the PATCHED build whose only change is that cap (1 GB;
                 oracle/Makefile, libmaul3d_ref_big.so) steps it, 30 steps.

  rain_10000_s3  the mixed rain field: 10,000 bodies (40 % spheres, 30 %
                 capsules, 30 % QuickHull hulls) falling onto a 255 x 255
                 heightfield, 4 substeps, the full 600 steps.

Every case records the hash after every step and checks that every step
advanced (no stall) and the scratch never overflowed.  Run from the
repository root (the 1000-tower case takes several minutes):

    python tests/golden/make_large_golden.py [case names, to regenerate only those]
"""
import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import ref  # noqa: E402

SCENE_CITY = 9
SCENE_RAIN = 10
# (name, scene, seed, param, substeps, steps, oracle build)
CASES = [
    ("city_300_s5", SCENE_CITY, 5, 300, 8, 30, "stock"),
    ("city_1000_s5", SCENE_CITY, 5, 1000, 8, 30, "big"),
    ("rain_10000_s3", SCENE_RAIN, 3, 10000, 4, 600, "stock"),
]


def main() -> None:
    only = set(sys.argv[1:])
    path = Path(__file__).with_name("large_traces.json")
    out = {"generator": "tests/golden/make_large_golden.py", "cases": []}
    if only and path.exists():
        # Regenerate the named cases only, keeping the others.
        out["cases"] = [c for c in json.loads(path.read_text())["cases"] if c["name"] not in only]
    for name, scene, seed, param, sub, steps, variant in CASES:
        if only and name not in only:
            continue
        w = ref.RefWorld.scene(scene, seed, param, variant=variant)
        h0 = w.hash()
        trace = w.trace(1.0 / 60.0, sub, steps)
        assert w.step_count() == steps, "the reference stalled"
        assert w.scratch_overflow() == 0
        out["cases"].append({
            "name": name, "scene": scene, "seed": seed, "param": param, "dt": 1.0 / 60.0,
            "substeps": sub, "steps": steps, "oracle": variant, "bodies": w.body_count(),
            "hash0": f"{h0:016x}", "trace": [f"{int(h):016x}" for h in trace],
        })
        w.destroy()
        print(name, out["cases"][-1]["trace"][-1], flush=True)
    order = [c[0] for c in CASES]
    out["cases"].sort(key=lambda c: order.index(c["name"]))
    path.write_text(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    main()
