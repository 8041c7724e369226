"""Oracle (test infrastructure only): the reference engine built from its
own C sources by oracle/Makefile, driven through its public API plus the
white-box capture harness (oracle/m3_oracle.c).

Parity is pinned: the same build reproduces every scene hash in the
reference's bench/pins.txt and its determinism gate hash
(tests/test_oracle_pins.py).  Only tests/, __graft_entry__.smoke() and
bench.py's CPU legs import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import importlib.util
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent


def _records():
    """The ctypes record types and value layouts (maul3d_b200/abi.py).

    abi.py depends on ctypes and numpy only.  When the package is already
    imported (the tests) its module is shared; otherwise the file is
    loaded on its own, so that driving the oracle never runs the
    package's __init__ and never maps this library's shared object (the
    reference arm of the bench loads the reference engine alone)."""
    mod = sys.modules.get("maul3d_b200.abi")
    if mod is not None:
        return mod
    spec = importlib.util.spec_from_file_location("m3_oracle_records",
                                                  REPO / "maul3d_b200" / "abi.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


abi = _records()
MANIFOLD, MAT3, TRANSFORM, VEC3 = abi.MANIFOLD, abi.MAT3, abi.TRANSFORM, abi.VEC3
WorldState, m3WorldId = abi.WorldState, abi.m3WorldId

REF_DIR = HERE / "_ref"
LIB_PATH = REF_DIR / "libmaul3d_ref.so"
BENCH_PATH = REF_DIR / "maul3d_bench"
DET_PATH = REF_DIR / "test_determinism"
# The reference's sources: M3_REFERENCE_SRC, else a checkout named
# `reference` beside this repository.  Absent on hosts that only use the
# prebuilt oracle/_ref.
REFERENCE_SRC = Path(os.environ.get("M3_REFERENCE_SRC") or (REPO.parent / "reference"))


def build(force: bool = False) -> bool:
    """Compile the oracle when the reference sources are present.

    Returns True when oracle/_ref holds a usable library afterwards.
    """
    if (REFERENCE_SRC / "src" / "solver.c").exists():
        cmd = ["make", "-C", str(HERE), f"REF={REFERENCE_SRC}", "-j8"]
        if force:
            subprocess.run(["make", "-C", str(HERE), "clean"], check=True)
        subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)
    return LIB_PATH.exists()


# The patched build for the largest world: the reference with only its
# step scratch cap raised from 1 << 28 to 1 << 30 bytes (oracle/Makefile).
BIG_LIB_PATH = REF_DIR / "libmaul3d_ref_big.so"
_libs: dict[str, C.CDLL] = {}


def lib(variant: str = "stock") -> C.CDLL:
    """The reference engine: "stock" (unmodified) or "big" (the patched
    scratch cap, for worlds the stock build stalls on)."""
    if variant not in _libs:
        path = LIB_PATH if variant == "stock" else BIG_LIB_PATH
        if not path.exists():
            build()
        h = C.CDLL(str(path))
        abi.bind_common(h)
        for name, n in (("m3o_copy_bodies", 5), ("m3o_copy_pairs", 2), ("m3o_copy_joints", 4)):
            fn = getattr(h, name)
            fn.argtypes = [m3WorldId] + [C.c_void_p] * n + [C.c_int32]
            fn.restype = C.c_int32
        h.m3o_copy_mass.argtypes = [m3WorldId] + [C.c_void_p] * 6 + [C.c_int32]
        h.m3o_copy_mass.restype = C.c_int32
        for name in ("m3o_body_max", "m3o_shape_max", "m3o_joint_max", "m3o_pair_count",
                     "m3o_scratch_overflow", "m3o_last_color_count", "m3o_pair_capacity"):
            getattr(h, name).argtypes = [m3WorldId]
            getattr(h, name).restype = C.c_int32
        h.m3o_step_count.argtypes = [m3WorldId]
        h.m3o_step_count.restype = C.c_uint64
        h.m3o_step_trace.argtypes = [m3WorldId, C.c_float, C.c_int32, C.c_int32, C.c_void_p]
        h.m3o_step_trace.restype = None
        h.m3o_copy_hull.argtypes = [m3WorldId, C.c_int32, C.c_void_p]
        h.m3o_copy_hull.restype = C.c_int32
        h.m3o_use_task_pool.argtypes = [m3WorldId, C.c_int32]
        h.m3o_use_task_pool.restype = C.c_int32
        _libs[variant] = h
    return _libs[variant]


class RefWorld:
    """One world inside the reference engine (the stock build unless
    `variant` says "big")."""

    def __init__(self, wid: m3WorldId, variant: str = "stock"):
        if wid.index1 == 0:
            raise RuntimeError("reference refused to create the world")
        self.id = wid
        self.lib = lib(variant)

    @classmethod
    def scene(cls, scene: int, seed: int = 0, param: int = 0,
              variant: str = "stock") -> "RefWorld":
        return cls(lib(variant).m3s_build(scene, seed, param), variant)

    def step(self, dt: float = 1.0 / 60.0, substeps: int = 4, steps: int = 1) -> None:
        self.lib.m3o_step_trace(self.id, dt, substeps, steps, None)

    def trace(self, dt: float, substeps: int, steps: int) -> np.ndarray:
        """Step and return the world hash after every step."""
        out = np.zeros(steps, np.uint64)
        self.lib.m3o_step_trace(self.id, dt, substeps, steps, out.ctypes.data)
        return out

    def hash(self) -> int:
        return int(self.lib.m3World_Hash(self.id))

    def destroy(self) -> None:
        self.lib.m3DestroyWorld(self.id)

    def body_count(self) -> int:
        return int(self.lib.m3o_body_max(self.id))

    def pair_count(self) -> int:
        return int(self.lib.m3o_pair_count(self.id))

    def scratch_overflow(self) -> int:
        return int(self.lib.m3o_scratch_overflow(self.id))

    def use_threads(self, threads: int) -> int:
        """Step on `threads` host threads through the reference's own task
        hooks (1: serial); returns the threads in use."""
        return int(self.lib.m3o_use_task_pool(self.id, threads))

    def step_count(self) -> int:
        return int(self.lib.m3o_step_count(self.id))

    def state(self) -> WorldState:
        n = self.body_count()
        xf = np.zeros(n, TRANSFORM)
        lin = np.zeros(n, VEC3)
        ang = np.zeros(n, VEC3)
        awake = np.zeros(n, np.uint8)
        sleep = np.zeros(n, np.float32)
        self.lib.m3o_copy_bodies(self.id, xf.ctypes.data, lin.ctypes.data, ang.ctypes.data,
                              awake.ctypes.data, sleep.ctypes.data, n)
        p = self.pair_count()
        keys = np.zeros(p, np.uint64)
        man = np.zeros(p, MANIFOLD)
        if p > 0:
            self.lib.m3o_copy_pairs(self.id, keys.ctypes.data, man.ctypes.data, p)
        return WorldState(xf, lin, ang, awake, sleep, keys, man)

    def mass(self) -> dict:
        n = self.body_count()
        out = {"invMass": np.zeros(n, np.float32), "invInertia": np.zeros(n, MAT3),
               "inertia": np.zeros(n, MAT3), "localCenter": np.zeros(n, VEC3),
               "minExtent": np.zeros(n, np.float32), "maxExtent": np.zeros(n, np.float32)}
        self.lib.m3o_copy_mass(self.id, *[out[k].ctypes.data for k in
                                       ("invMass", "invInertia", "inertia", "localCenter",
                                        "minExtent", "maxExtent")], n)
        return out


def run_bench(steps: int = 300, timeout: float = 600.0) -> dict[str, str]:
    """Run the reference's own bench harness; scene name -> printed hash."""
    out = subprocess.run([str(BENCH_PATH), str(steps)], capture_output=True, text=True,
                         timeout=timeout, check=True).stdout
    hashes = {}
    for line in out.splitlines():
        parts = line.split()
        if len(parts) >= 2 and parts[0] == "M3_BENCH" and "hash=" in line:
            hashes[parts[1]] = line.split("hash=")[1].split()[0]
    return hashes
