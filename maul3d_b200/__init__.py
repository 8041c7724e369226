"""maul3d_b200: the Maul3D step path on NVIDIA B200 (sm_100a).

Python host mirror of the reference engine's public API for the step
path (include/maul3d/world.h: m3World_Step, m3World_Hash), bound to the
in-tree shared library libmaul3d_b200.so over its C ABI.  There is no
Python or CPU fallback: if the library is missing, importing this
package raises, and stepping without a CUDA device raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import abi
from .abi import MANIFOLD, TRANSFORM, VEC3, MAT3, WorldState, m3WorldId

_LIB_PATH = Path(__file__).resolve().parent / "libmaul3d_b200.so"

M3GPU_OK = 0
M3GPU_ERR_INVALID = 1
M3GPU_ERR_CUDA = 2
M3GPU_ERR_CAPACITY = 3
M3GPU_ERR_UNSUPPORTED = 4
M3GPU_ERR_NO_DEVICE = 5


class M3GpuError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"maul3d_b200 error {code}: {message}")
        self.code = code


def _load() -> C.CDLL:
    if not _LIB_PATH.exists():
        raise ImportError(
            f"{_LIB_PATH} is missing: build it with `python maul3d_b200/build.py` "
            "(the CUDA path has no CPU fallback)")
    lib = C.CDLL(str(_LIB_PATH))
    abi.bind_common(lib)
    lib.m3gpu_last_error.restype = C.c_int32
    lib.m3gpu_last_error_message.restype = C.c_char_p
    lib.m3gpu_step_worlds.argtypes = [C.POINTER(m3WorldId), C.c_int32, C.c_float, C.c_int32, C.c_int32]
    lib.m3gpu_step_worlds.restype = C.c_int32
    lib.m3gpu_hash_worlds.argtypes = [C.POINTER(m3WorldId), C.c_int32, C.POINTER(C.c_uint64)]
    lib.m3gpu_hash_worlds.restype = C.c_int32
    lib.m3gpu_synchronize.restype = C.c_int32
    lib.m3gpu_launch_count.restype = C.c_int64
    lib.m3gpu_last_step_ms.restype = C.c_float
    lib.m3gpu_body_max.argtypes = [m3WorldId]
    lib.m3gpu_body_max.restype = C.c_int32
    lib.m3gpu_pair_count.argtypes = [m3WorldId]
    lib.m3gpu_pair_count.restype = C.c_int32
    for name, n in (("m3gpu_copy_bodies", 5), ("m3gpu_copy_pairs", 2), ("m3gpu_copy_joints", 4)):
        fn = getattr(lib, name)
        fn.argtypes = [m3WorldId] + [C.c_void_p] * n + [C.c_int32]
        fn.restype = C.c_int32
    lib.m3gpu_copy_mass.argtypes = [m3WorldId] + [C.c_void_p] * 6 + [C.c_int32]
    lib.m3gpu_copy_mass.restype = C.c_int32
    abi.bind_snapshot(lib)
    abi.bind_replay(lib)
    lib.m3gpu_serve_create.argtypes = [C.c_int64, C.c_int32]
    lib.m3gpu_serve_create.restype = C.c_void_p
    lib.m3gpu_serve_destroy.argtypes = [C.c_void_p]
    lib.m3gpu_serve_destroy.restype = None
    lib.m3gpu_serve_submit.argtypes = [C.c_void_p, C.c_void_p, C.c_int32]
    lib.m3gpu_serve_submit.restype = C.c_int64
    lib.m3gpu_serve_tick.argtypes = [C.c_void_p]
    lib.m3gpu_serve_tick.restype = C.c_int32
    lib.m3gpu_serve_poll.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32]
    lib.m3gpu_serve_poll.restype = C.c_int32
    lib.m3gpu_serve_active.argtypes = [C.c_void_p]
    lib.m3gpu_serve_active.restype = C.c_int32
    lib.m3gpu_serve_stats.argtypes = [C.c_void_p, C.POINTER(abi.m3gpuServeStats)]
    lib.m3gpu_serve_stats.restype = C.c_int32
    lib.m3gpu_step_worlds_commands.argtypes = [C.POINTER(abi.m3WorldId), C.c_int32, C.c_float,
                                               C.c_int32, C.POINTER(abi.m3gpuBodyCommand),
                                               C.c_int32]
    lib.m3gpu_step_worlds_commands.restype = C.c_int32
    lib.m3gpu_get_packing.argtypes = [C.POINTER(abi.m3gpuPacking)]
    lib.m3gpu_get_packing.restype = C.c_int32
    lib.m3gpu_set_packing.argtypes = [C.POINTER(abi.m3gpuPacking)]
    lib.m3gpu_set_packing.restype = C.c_int32
    lib.m3gpu_autotune_packing.argtypes = [C.POINTER(abi.m3WorldId), C.c_int32, C.c_float,
                                           C.c_int32, C.c_int32, C.POINTER(abi.m3gpuPacking),
                                           C.POINTER(C.c_float)]
    lib.m3gpu_autotune_packing.restype = C.c_int32
    lib.m3gpu_autotune_trials.argtypes = [C.POINTER(abi.m3gpuPackingTrial), C.c_int32]
    lib.m3gpu_autotune_trials.restype = C.c_int32
    for name in ("m3gpu_slots_reserve", "m3gpu_slot_save", "m3gpu_slot_restore"):
        getattr(lib, name).argtypes = [abi.m3WorldId, C.c_int32]
        getattr(lib, name).restype = C.c_int32
    lib.m3gpu_set_device.argtypes = [C.c_int32]
    lib.m3gpu_set_device.restype = C.c_int32
    for name in ("m3gpu_reserve_worlds", "m3gpu_upload_worlds"):
        getattr(lib, name).argtypes = [C.POINTER(m3WorldId), C.c_int32]
        getattr(lib, name).restype = C.c_int32
    lib.m3gpu_world_image_bytes.argtypes = [m3WorldId]
    lib.m3gpu_world_image_bytes.restype = C.c_int64
    lib.m3gpu_uploaded_bytes.argtypes = []
    lib.m3gpu_uploaded_bytes.restype = C.c_int64
    lib.m3gpu_kernel_ms.argtypes = [C.POINTER(C.c_float)]
    lib.m3gpu_kernel_ms.restype = C.c_int32
    lib.m3gpu_world_stats.argtypes = [m3WorldId, C.POINTER(C.c_uint64)]
    lib.m3gpu_world_stats.restype = C.c_int32
    lib.m3gpu_world_phase_cycles.argtypes = [m3WorldId, C.POINTER(C.c_uint64)]
    lib.m3gpu_world_phase_cycles.restype = C.c_int32
    lib.m3gpu_flush_trees.argtypes = [C.POINTER(m3WorldId), C.c_int32]
    lib.m3gpu_flush_trees.restype = C.c_int32
    lib.m3gpu_set_wide_min_shapes.argtypes = [C.c_int32]
    lib.m3gpu_set_wide_min_shapes.restype = C.c_int32
    return lib


lib = _load()


def last_error() -> tuple[int, str]:
    return int(lib.m3gpu_last_error()), lib.m3gpu_last_error_message().decode()


def _check(rc: int) -> None:
    if rc != M3GPU_OK:
        code, msg = last_error()
        raise M3GpuError(rc, msg)


def _ids(worlds) -> "C.Array":
    if isinstance(worlds, WorldBatch):
        return worlds.ids
    arr = (m3WorldId * len(worlds))()
    for i, w in enumerate(worlds):
        arr[i] = w.id
    return arr


class WorldBatch:
    """A fixed list of worlds with its id array built once, for callers
    that step and hash the same batch many times."""

    def __init__(self, worlds):
        self.worlds = list(worlds)
        self.ids = (m3WorldId * len(self.worlds))()
        for i, w in enumerate(self.worlds):
            self.ids[i] = w.id
        self.hashes = np.zeros(len(self.worlds), dtype=np.uint64)

    def __len__(self) -> int:
        return len(self.worlds)

    def __iter__(self):
        return iter(self.worlds)


class World:
    """One world living in this library (host image + HBM slab)."""

    def __init__(self, wid: m3WorldId):
        if wid.index1 == 0:
            code, msg = last_error()
            raise M3GpuError(code or M3GPU_ERR_INVALID, msg)
        self.id = wid

    @classmethod
    def scene(cls, scene: int, seed: int = 0, param: int = 0) -> "World":
        """Build one of the seeded synthetic scenes (csrc/scenes.c)."""
        return cls(lib.m3s_build(scene, seed, param))

    def step(self, dt: float = 1.0 / 60.0, substeps: int = 4, steps: int = 1) -> None:
        _check(lib.m3gpu_step_worlds(_ids([self]), 1, dt, substeps, steps))

    def hash(self) -> int:
        h = int(lib.m3World_Hash(self.id))
        code, msg = last_error()
        if code != M3GPU_OK:
            raise M3GpuError(code, msg)
        return h

    def destroy(self) -> None:
        lib.m3DestroyWorld(self.id)

    def reserve_slots(self, slots: int) -> None:
        """Device snapshot slots in HBM (m3gpu_slots_reserve)."""
        _check(lib.m3gpu_slots_reserve(self.id, slots))

    def save_slot(self, slot: int) -> None:
        _check(lib.m3gpu_slot_save(self.id, slot))

    def restore_slot(self, slot: int) -> None:
        _check(lib.m3gpu_slot_restore(self.id, slot))

    def body_count(self) -> int:
        return int(lib.m3gpu_body_max(self.id))

    def state(self) -> WorldState:
        n = self.body_count()
        xf = np.zeros(n, TRANSFORM)
        lin = np.zeros(n, VEC3)
        ang = np.zeros(n, VEC3)
        awake = np.zeros(n, np.uint8)
        sleep = np.zeros(n, np.float32)
        got = lib.m3gpu_copy_bodies(self.id, xf.ctypes.data, lin.ctypes.data, ang.ctypes.data,
                                    awake.ctypes.data, sleep.ctypes.data, n)
        if got < 0:
            code, msg = last_error()
            raise M3GpuError(code or M3GPU_ERR_INVALID,
                             f"body readback failed ({n} bodies asked): {msg}")
        p = int(lib.m3gpu_pair_count(self.id))
        keys = np.zeros(max(p, 0), np.uint64)
        man = np.zeros(max(p, 0), MANIFOLD)
        if p > 0:
            lib.m3gpu_copy_pairs(self.id, keys.ctypes.data, man.ctypes.data, p)
        return WorldState(xf, lin, ang, awake, sleep, keys, man)

    def mass(self) -> dict:
        n = self.body_count()
        out = {"invMass": np.zeros(n, np.float32), "invInertia": np.zeros(n, MAT3),
               "inertia": np.zeros(n, MAT3), "localCenter": np.zeros(n, VEC3),
               "minExtent": np.zeros(n, np.float32), "maxExtent": np.zeros(n, np.float32)}
        lib.m3gpu_copy_mass(self.id, *[out[k].ctypes.data for k in
                                       ("invMass", "invInertia", "inertia", "localCenter",
                                        "minExtent", "maxExtent")], n)
        return out


def step_worlds(worlds, dt: float = 1.0 / 60.0, substeps: int = 4, steps: int = 1) -> None:
    """Step many worlds in one batched launch sequence (one block per world)."""
    _check(lib.m3gpu_step_worlds(_ids(worlds), len(worlds), dt, substeps, steps))


def step_worlds_commands(worlds, commands, dt: float = 1.0 / 60.0, substeps: int = 4) -> None:
    """Body commands on the device, then one step (m3gpu_step_worlds_commands).
    `commands`: (world index, op, m3BodyId, (x, y, z)) tuples."""
    arr = (abi.m3gpuBodyCommand * max(len(commands), 1))()
    for k, (wi, op, body, v) in enumerate(commands):
        arr[k] = abi.m3gpuBodyCommand(wi, op, body, abi.m3Vec3(*v))
    _check(lib.m3gpu_step_worlds_commands(_ids(worlds), len(worlds), dt, substeps, arr,
                                          len(commands)))


def get_packing() -> dict:
    """The batched step's packing in use (m3gpu_get_packing)."""
    p = abi.m3gpuPacking()
    _check(lib.m3gpu_get_packing(C.byref(p)))
    return p.as_dict()


def set_packing(packing: dict) -> None:
    """Selects a packing (m3gpu_set_packing): {"min_shapes": [a, b],
    "threads": [t0, t1, t2], "smem_bytes": [s0, s1, s2]}."""
    _check(lib.m3gpu_set_packing(C.byref(abi.m3gpuPacking.from_dict(packing))))


def autotune_packing(worlds, dt: float = 1.0 / 60.0, substeps: int = 4,
                     steps: int = 24) -> tuple[dict, float]:
    """Steps the worlds `steps` times while timing candidate packings
    (m3gpu_autotune_packing); returns the packing left in use and its
    prepare + substep device time per step in milliseconds."""
    p = abi.m3gpuPacking()
    ms = C.c_float(0.0)
    _check(lib.m3gpu_autotune_packing(_ids(worlds), len(worlds), dt, substeps, steps,
                                      C.byref(p), C.byref(ms)))
    return p.as_dict(), float(ms.value)


def autotune_trials() -> list[dict]:
    """The last autotuning's candidates in order (m3gpu_autotune_trials):
    packing, its step's prepare + substep ms, the mean of the steps beside
    it under the packing then in use, and whether it was adopted."""
    n = int(lib.m3gpu_autotune_trials(None, 0))
    arr = (abi.m3gpuPackingTrial * max(n, 1))()
    n = int(lib.m3gpu_autotune_trials(arr, n))
    return [{"packing": t.packing.as_dict(), "ms": float(t.ms),
             "baseline_ms": float(t.baselineMs), "adopted": bool(t.adopted)} for t in arr[:n]]


def hash_worlds(worlds) -> np.ndarray:
    """World hashes computed on the device, one thread block per world.
    For a WorldBatch the result is written into (and returned as) its
    `hashes` array."""
    out = worlds.hashes if isinstance(worlds, WorldBatch) else np.zeros(len(worlds), np.uint64)
    _check(lib.m3gpu_hash_worlds(_ids(worlds), len(worlds),
                                 out.ctypes.data_as(C.POINTER(C.c_uint64))))
    return out


def flush_trees(worlds) -> None:
    """Replay every recorded tree move of the worlds and wait (the trees
    are then current, as a snapshot needs them)."""
    _check(lib.m3gpu_flush_trees(_ids(worlds), len(worlds)))


def synchronize() -> None:
    _check(lib.m3gpu_synchronize())


def launch_count() -> int:
    return int(lib.m3gpu_launch_count())


def last_step_ms() -> float:
    return float(lib.m3gpu_last_step_ms())


def set_device(device: int) -> None:
    _check(lib.m3gpu_set_device(device))


def reserve_worlds(worlds) -> None:
    _check(lib.m3gpu_reserve_worlds(_ids(worlds), len(worlds)))


def upload_worlds(worlds) -> None:
    _check(lib.m3gpu_upload_worlds(_ids(worlds), len(worlds)))


def image_bytes(world) -> int:
    return int(lib.m3gpu_world_image_bytes(world.id))


def uploaded_bytes() -> int:
    """Host-to-device bytes copied by world uploads so far."""
    return int(lib.m3gpu_uploaded_bytes())


STAGES = ("broad", "narrow", "prepare", "substep", "finish")


def kernel_ms() -> dict[str, float]:
    """Device milliseconds of the last batched step call per stage:
    broad (bounds, pairs), narrow (narrowphase), prepare (islands,
    colouring, rows), substep (the substep loop, restitution, store) and
    finish (continuous, sleep), each summed over the call's steps;
    collide = broad + narrow."""
    out = (C.c_float * len(STAGES))()
    _check(lib.m3gpu_kernel_ms(out))
    ms = {name: float(out[k]) for k, name in enumerate(STAGES)}
    ms["collide"] = ms["broad"] + ms["narrow"]
    return ms


def set_wide_min_shapes(shapes: int) -> int:
    """A single world with at least `shapes` shape slots steps its
    substep loop over the whole grid; returns the previous threshold."""
    return int(lib.m3gpu_set_wide_min_shapes(shapes))


def counters(world) -> dict[str, int]:
    """m3World_GetCounters of one world, as a dict."""
    c = lib.m3World_GetCounters(world.id)
    return {name: getattr(c, name) for name, _ in c._fields_}


def profile(world) -> dict[str, float]:
    """m3World_GetProfile of one world (milliseconds of its last step)."""
    p = lib.m3World_GetProfile(world.id)
    return {name: getattr(p, name) for name, _ in p._fields_}


PHASES = ("islands", "prepare", "colour+movers", "integrate_v", "warm_start", "bias_solve",
          "integrate_p", "relax", "store", "continuous", "sleep", "bounds", "sweep_sort",
          "pair_count", "pair_fill", "tree_moves")


def world_phase_cycles(world) -> np.ndarray:
    """Device clock cycles the world's block spent per step phase (PHASES;
    the last entry counts the broadphase tree's leaf moves replayed)."""
    out = (C.c_uint64 * 16)()
    _check(lib.m3gpu_world_phase_cycles(world.id, out))
    return np.array(list(out), dtype=np.uint64)


def world_stats(world) -> np.ndarray:
    """Work counters: mover-substeps, contact-row-substeps, joint-row-substeps,
    candidate pairs, steps, body slots."""
    out = (C.c_uint64 * 6)()
    _check(lib.m3gpu_world_stats(world.id, out))
    return np.array(list(out), dtype=np.uint64)


class Server:
    """Batched serving of replay containers (snapshot + journal): submit,
    tick until idle, poll the final hashes (m3gpu_serve_*)."""

    def __init__(self, device_budget: int = 64 << 30, max_active: int = 4096):
        self.handle = lib.m3gpu_serve_create(device_budget, max_active)
        if not self.handle:
            raise M3GpuError(*last_error())

    def submit(self, container: bytes) -> int:
        # The server copies what it keeps: the bytes are passed in place.
        ticket = int(lib.m3gpu_serve_submit(self.handle, bytes(container), len(container)))
        if ticket < 0:
            raise M3GpuError(*last_error())
        return ticket

    def tick(self) -> int:
        """One frame for every active request; returns queued + active."""
        n = int(lib.m3gpu_serve_tick(self.handle))
        if n < 0:
            raise M3GpuError(-n, last_error()[1])
        return n

    def active(self) -> int:
        return int(lib.m3gpu_serve_active(self.handle))

    def stats(self) -> dict:
        """Counters and host times since creation (m3gpu_serve_stats)."""
        out = abi.m3gpuServeStats()
        _check(lib.m3gpu_serve_stats(self.handle, C.byref(out)))
        return {name: getattr(out, name) for name, _ in out._fields_ if name != "reserved"}

    def poll(self, capacity: int = 4096):
        """Finished requests: arrays of tickets, hashes and statuses."""
        t = np.zeros(capacity, np.int64)
        h = np.zeros(capacity, np.uint64)
        st = np.zeros(capacity, np.int32)
        n = int(lib.m3gpu_serve_poll(self.handle, t.ctypes.data, h.ctypes.data, st.ctypes.data,
                                     capacity))
        return t[:n], h[:n], st[:n]

    def run(self) -> dict[int, tuple[int, int]]:
        """Tick until idle; {ticket: (hash, status)} of everything finished."""
        out = {}
        while True:
            left = self.tick()
            t, h, st = self.poll()
            for k in range(len(t)):
                out[int(t[k])] = (int(h[k]), int(st[k]))
            if left == 0:
                t, h, st = self.poll()
                for k in range(len(t)):
                    out[int(t[k])] = (int(h[k]), int(st[k]))
                return out

    def close(self) -> None:
        if self.handle:
            lib.m3gpu_serve_destroy(self.handle)
            self.handle = None


def snapshot(world) -> bytes:
    """The world's snapshot bytes (m3World_Snapshot)."""
    n = int(lib.m3World_SnapshotSize(world.id))
    if n < 0:
        raise M3GpuError(*last_error())
    buf = (C.c_uint8 * n)()
    if lib.m3World_Snapshot(world.id, buf, n) != n:
        raise M3GpuError(*last_error())
    return bytes(buf)
