"""Packing of a batch onto the SMs, and its autotuner (needs a B200).

The batched step splits its worlds into three size classes by shape
slots; each class runs one of three kernel variants (512, 256 or 128
threads per world: one, two or four worlds resident per SM) with a
shared-memory budget for its tables.  The packing changes where rows run,
never their arithmetic: under every packing below, including ones that
put every world on one variant and ones that keep every table in global
memory, each world's hash must equal the reference engine's after every
step.  The autotuner's steps are real steps: a batch tuned for N steps
ends on the same hashes as the same batch stepped N times.
"""
import pytest

from conftest import cuda_available
from maul3d_b200.abi import SCENE_BOUNCE, SCENE_PLANK, SCENE_TOWERS, SCENE_UNEVEN

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")]

DT = 1.0 / 60.0
SUB = 4
STEPS = 16

# Uneven worlds across the three default classes (up to 160 shape slots,
# 161-768, above 768), the overflow colour (plank), restitution (bounce)
# and breaking fixed joints (towers).
SPECS = ([(SCENE_UNEVEN, 300 + i, n) for i, n in enumerate([32, 90, 150, 400, 700, 1100, 2048])] +
         [(SCENE_PLANK, 311, 30), (SCENE_BOUNCE, 312, 60), (SCENE_TOWERS, 313, 6)])

DEFAULT = {"min_shapes": [769, 161], "threads": [512, 256, 128],
           "smem_bytes": [200 * 1024, 110 * 1024, 54 * 1024]}
PACKINGS = {
    "default": DEFAULT,
    # every world in class 2, 128 threads per world
    "all_128": {"min_shapes": [1 << 30, (1 << 30) - 1], "threads": [512, 256, 128],
                "smem_bytes": DEFAULT["smem_bytes"]},
    # every world in class 0, 512 threads per world
    "all_512": {"min_shapes": [2, 1], "threads": [512, 256, 128],
                "smem_bytes": DEFAULT["smem_bytes"]},
    # every table (body cache included) in global memory
    "no_shared": {"min_shapes": [769, 161], "threads": [512, 256, 128], "smem_bytes": [0, 0, 0]},
    # variants swapped between the classes, budgets tight
    "swapped": {"min_shapes": [400, 100], "threads": [128, 512, 256],
                "smem_bytes": [54 * 1024, 0, 110 * 1024]},
}


@pytest.fixture(scope="module")
def reference_traces(oracle):
    """Every world's hash after each step, from the reference engine."""
    traces = []
    for spec in SPECS:
        r = oracle.RefWorld.scene(*spec)
        trace = []
        for _ in range(STEPS):
            r.step(DT, SUB, 1)
            trace.append(r.hash())
        r.destroy()
        traces.append(trace)
    return traces


@pytest.fixture
def restore_packing(m3):
    previous = m3.get_packing()
    yield
    m3.set_packing(previous)


@pytest.mark.parametrize("name", sorted(PACKINGS))
def test_every_packing_matches_the_reference(m3, reference_traces, restore_packing, name):
    m3.set_packing(PACKINGS[name])
    assert m3.get_packing() == PACKINGS[name]
    worlds = [m3.World.scene(*spec) for spec in SPECS]
    for step in range(STEPS):
        m3.step_worlds(worlds, DT, SUB, 1)
        got = [int(h) for h in m3.hash_worlds(worlds)]
        want = [t[step] for t in reference_traces]
        bad = [SPECS[i] for i in range(len(SPECS)) if got[i] != want[i]]
        assert not bad, f"packing {name}, step {step + 1}: {bad}"
    for w in worlds:
        w.destroy()


def test_autotuned_steps_are_real_steps(m3, reference_traces, restore_packing):
    """The tuner's steps (candidates between steps of the packing in use)
    leave every world where plain steps would, and the packing it returns
    is the one left in use."""
    m3.set_packing(DEFAULT)
    worlds = [m3.World.scene(*spec) for spec in SPECS]
    packing, ms = m3.autotune_packing(worlds, DT, SUB, STEPS)
    assert m3.get_packing() == packing
    assert ms > 0.0
    # 16 steps: the first under the default, then each candidate between
    # two steps of the packing in use (7 candidates at most).
    trials = m3.autotune_trials()
    assert 1 <= len(trials) <= (STEPS - 1) // 2
    adopted = [t["packing"] for t in trials if t["adopted"]]
    assert packing == (adopted[-1] if adopted else DEFAULT)
    for t in trials:
        assert t["ms"] > 0.0 and t["baseline_ms"] > 0.0
        assert t["adopted"] == (t["ms"] < 0.97 * t["baseline_ms"])
    got = [int(h) for h in m3.hash_worlds(worlds)]
    assert got == [t[STEPS - 1] for t in reference_traces]
    # Fewer than 3 steps only step, under the packing in use.
    assert m3.autotune_packing(worlds, DT, SUB, 2)[0] == packing
    assert m3.autotune_trials() == []
    for w in worlds:
        w.destroy()


def test_packing_change_reclassifies_a_prepared_batch(m3, reference_traces, restore_packing):
    """A batch prepared under one packing and stepped on under another
    (the same world list, so no fresh preparation) follows the new one
    and still matches the reference."""
    m3.set_packing(DEFAULT)
    worlds = [m3.World.scene(*spec) for spec in SPECS]
    names = ["default", "all_128", "no_shared", "swapped", "all_512"]
    for step in range(STEPS):
        m3.set_packing(PACKINGS[names[step % len(names)]])
        m3.step_worlds(worlds, DT, SUB, 1)
    got = [int(h) for h in m3.hash_worlds(worlds)]
    assert got == [t[STEPS - 1] for t in reference_traces]
    for w in worlds:
        w.destroy()


def test_world_beyond_the_body_cache_in_a_batch(m3, oracle, restore_packing):
    """A 4,600-body world stepped in a batch (not alone, so not on the
    wide path): its 52-byte-a-body cache would pass the 200 KB shared-memory
    limit, so only its velocities are cached; a world that needs more than
    even those (the 0-byte budget) keeps everything in global memory.  Both
    match the reference every step."""
    specs = [(SCENE_UNEVEN, 331, 4600), (SCENE_UNEVEN, 332, 300)]
    refs = [oracle.RefWorld.scene(*spec) for spec in specs]
    traces = []
    for r in refs:
        trace = []
        for _ in range(8):
            r.step(DT, SUB, 1)
            trace.append(r.hash())
        traces.append(trace)
        r.destroy()
    for packing in (DEFAULT, PACKINGS["no_shared"]):
        m3.set_packing(packing)
        worlds = [m3.World.scene(*spec) for spec in specs]
        for step in range(8):
            m3.step_worlds(worlds, DT, SUB, 1)
            got = [int(h) for h in m3.hash_worlds(worlds)]
            assert got == [t[step] for t in traces], f"step {step + 1}"
        for w in worlds:
            w.destroy()
