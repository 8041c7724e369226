"""The C ABI: the in-tree library loads and exports every entry point
include/maul3d_b200.h declares (no device calls)."""
import ctypes as C
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "maul3d_b200.h").read_text()
    return sorted(set(re.findall(r"M3GPU_API\s+[^;(]*?\b(m3\w+)\s*\(", text)))


def test_header_declares_the_drop_in_entries():
    names = declared_symbols()
    for required in ("m3World_Step", "m3World_Hash", "m3CreateWorld", "m3CreateBody",
                     "m3CreateBoxShape", "m3gpu_step_worlds", "m3gpu_hash_worlds"):
        assert required in names


def test_library_exports_every_declared_symbol(m3):
    lib = C.CDLL(str(ROOT / "maul3d_b200" / "libmaul3d_b200.so"))
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_library_links_no_reference_code():
    # The product never links the oracle: no reference-only internals.
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only",
                          str(ROOT / "maul3d_b200" / "libmaul3d_b200.so")],
                         capture_output=True, text=True, check=True).stdout
    assert "m3StepInternal" not in out
    assert "m3o_" not in out


def test_packing_is_checked_and_kept(m3):
    """m3gpu_set_packing refuses impossible packings and keeps the last
    valid one (host state only: no device call)."""
    import pytest
    before = m3.get_packing()
    try:
        good = {"min_shapes": [500, 100], "threads": [256, 128, 512],
                "smem_bytes": [100000, 0, 204800]}
        m3.set_packing(good)
        assert m3.get_packing() == good
        for bad in ({"min_shapes": [100, 100], "threads": [512, 256, 128], "smem_bytes": [0, 0, 0]},
                    {"min_shapes": [100, 0], "threads": [512, 256, 128], "smem_bytes": [0, 0, 0]},
                    {"min_shapes": [500, 100], "threads": [512, 64, 128], "smem_bytes": [0, 0, 0]},
                    {"min_shapes": [500, 100], "threads": [512, 256, 128],
                     "smem_bytes": [0, -1, 0]},
                    {"min_shapes": [500, 100], "threads": [512, 256, 128],
                     "smem_bytes": [0, 0, 204801]}):
            with pytest.raises(m3.M3GpuError):
                m3.set_packing(bad)
            assert m3.get_packing() == good
    finally:
        m3.set_packing(before)
