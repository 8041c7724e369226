"""Shared test setup: the `gpu` marker, import paths, and the oracle.

`-m gpu` tests need a CUDA device; everything else runs on the CPU.
The oracle (oracle/_ref, the reference engine built from its own
sources) is built here on first use when the reference sources are
present, and otherwise taken prebuilt.
"""
import json
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


# Number of golden trace cases in tests/golden/traces.json.
GOLDEN_CASES = len(json.loads((ROOT / "tests" / "golden" / "traces.json").read_text())["cases"])


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import ref
    if not ref.build():
        pytest.skip("oracle library unavailable (no reference sources, no prebuilt oracle/_ref)")
    return ref


@pytest.fixture(scope="session")
def golden():
    return json.loads((ROOT / "tests" / "golden" / "traces.json").read_text())


@pytest.fixture(scope="session")
def m3():
    import maul3d_b200
    return maul3d_b200


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
