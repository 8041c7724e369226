"""Benchmark: bit-exact body-substeps/s of the batched device step.

Workload (default): the batched uneven-worlds configuration -- 4096
independent worlds per GPU, dynamic body counts log-uniform in
[32, 2048], each world 8-high box stacks (half extent U[0.25, 0.75]),
loose spheres and three revolute chains of 8 capsules (r 0.1,
half-height 0.4) hung from static anchors; dt 1/60, 4 substeps.  The
worlds are seeded synthetic scenes built through the library's
reference-compatible creation API (maul3d_b200/csrc/scenes.c).

One "step" = one m3World_Step of every world in the batch, everything
the reference's step does included (the broadphase tree it keeps as
snapshot state too).  The metric counts alive dynamic bodies x substeps
x steps over all worlds and all ranks, divided by the max-over-ranks
device time of exactly K steps.  First the packing autotuner steps a
copy of the batch (the same worlds, built apart) --tune-steps times, real
untimed steps that try packings of the worlds onto the SMs; the timed
batch, built fresh, runs under the packing it leaves (`packing`).

Lines printed by rank 0 (one JSON object):
  value     device-resident throughput (CUDA events around K steps);
  e2e       the same metric through the C ABI from host-built worlds:
            the H2D upload of every world image, K steps and a D2H read
            of every world's hash after each step, inside the timed
            region;
  roofline  the dominant kernel's algorithmic bytes / its device time,
            against the measured HBM copy bandwidth;
  plain_gpu the one-world-per-launch path on a sample of the worlds;
  cpu_baseline  the reference engine (oracle/_ref, built from its own
            sources) on the host cores, stepping a bounded sample of the
            same worlds for the same W+K steps, every sampled world's
            hash checked against the device's;
  serving   the serving path: replay containers (snapshot + journal of
            impulse frames) of worlds of 200-5000 bodies (boxes, spheres,
            16-point hulls) arriving as a Poisson process at 100-20,000
            requests/s, p50/p99 latency from arrival to final hash and
            throughput, a run with every request at once, and the
            reference's restore + replay of the same containers on the
            host cores, every answer compared.

Multi-GPU: one process per GPU (torchrun), each rank its own 4096
worlds (weak scaling), no collective on the data path; the only NCCL
calls are the timing barrier and the max/sum reductions of the result.

--impl reference runs the reference engine alone on the host cores
(all threads) for the same metric and config.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "bit-exact body-substeps/s"
UNIT = "body-substeps/s"
DT = 1.0 / 60.0
SCENE_UNEVEN = 2
SCENE_TERRAIN = 5

# Algorithmic bytes per unit of work of the substep loop (the
# reference's record layouts): per moving body per substep, integrate
# velocities 141 B + integrate positions 173 B; per contact row per
# substep 3 passes x (456 B record + 2 x 48 B v,w + 2 x 28 B dp,dq); per
# joint row per substep 3 x (472 + 152).
# DRAM bytes (read + write) of one step's m3SubstepKernel launches (the
# three size classes; the 4th step from creation) on the default
# workload, from ncu (dram__bytes_read.sum + dram__bytes_write.sum, one
# pass; profiles/m3SubstepKernel_uneven4096.txt gives the command):
# 902.5 + 677.7 MB (512-thread class), 381.8 + 391.5 MB (256), 80.5 +
# 102.4 MB (128).  Reported for that workload only.
SUBSTEP_TRAFFIC_DEFAULT = (902.5 + 677.7 + 381.8 + 391.5 + 80.5 + 102.4) * 1e6
BYTES_PER_MOVER_SUBSTEP = 314
BYTES_PER_CONTACT_SUBSTEP = 3 * (456 + 2 * 48 + 2 * 28)
BYTES_PER_JOINT_SUBSTEP = 3 * (472 + 152)


def default_workload(args) -> bool:
    return (args.worlds, args.lo, args.hi, args.substeps, args.seed) == (4096, 32, 2048, 4, 20261203)


def env_int(name: str, default: int) -> int:
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def world_sizes(lib, seed: int, count: int, lo: int, hi: int) -> list[int]:
    return [int(lib.m3s_uneven_size(seed, i, lo, hi)) for i in range(count)]


def measured_peaks() -> tuple[float, str]:
    path = ROOT / "MEASURED_PEAKS.json"
    try:
        data = json.loads(path.read_text())
        return float(data["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self) -> None:
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200", "-f", self.path],
                stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict | None:
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        try:
            for line in Path(self.path).read_text().splitlines():
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
            os.unlink(self.path)
        except Exception:
            return None
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def build_worlds(m3, sizes: list[int], seeds):
    """Seeded uneven worlds; `seeds` is a list (one per world) or a base
    seed (world i gets seed + i)."""
    if isinstance(seeds, int):
        seeds = [seeds + i for i in range(len(sizes))]
    return [m3.World.scene(SCENE_UNEVEN, s, n) for s, n in zip(seeds, sizes)]


def body_substeps(sizes: list[int], substeps: int, steps: int) -> int:
    return sum(sizes) * substeps * steps


# ---------------------------------------------------------------------------
# Reference engine on the host cores (oracle/_ref).  Worlds live in waves
# of at most 64 (the reference's world table); each wave steps on
# `threads` host threads, one world per task.  Only m3World_Step calls
# are timed.
# ---------------------------------------------------------------------------
def reference_run(sizes, seed, substeps, steps, threads, time_budget_s, want_hashes=False):
    from oracle import ref
    lib = ref.lib()
    done_bs = 0
    busy = 0.0
    hashes = {}
    index = 0
    t_start = time.perf_counter()
    while index < len(sizes):
        wave = list(range(index, min(index + 64, len(sizes))))
        index = wave[-1] + 1
        worlds = [ref.RefWorld.scene(SCENE_UNEVEN, seed + i, sizes[i]) for i in wave]
        queue = list(range(len(wave)))
        lock = threading.Lock()

        def worker():
            while True:
                with lock:
                    if not queue:
                        return
                    k = queue.pop(0)
                lib.m3o_step_trace(worlds[k].id, DT, substeps, steps, None)

        t0 = time.perf_counter()
        pool = [threading.Thread(target=worker) for _ in range(threads)]
        for t in pool:
            t.start()
        for t in pool:
            t.join()
        busy += time.perf_counter() - t0
        for k, i in enumerate(wave):
            if want_hashes:
                hashes[i] = worlds[k].hash()
            worlds[k].destroy()
        done_bs += body_substeps([sizes[i] for i in wave], substeps, steps)
        if time.perf_counter() - t_start > time_budget_s:
            break
    return done_bs, busy, hashes, index


def run_reference_arm(args) -> None:
    """The reference engine alone (oracle/_ref, built from its own
    sources; this library is never loaded) on every host thread, for the
    device arm's metric and workload: all of the batch's worlds, in waves
    of at most 64 (the reference's world table).  Per wave the worlds are
    built (untimed), stepped W warm-up steps (untimed), then K timed
    steps, one world per task, largest first; the value is the K steps'
    body-substeps of every world over the summed wall time of the waves'
    timed phases."""
    rank = env_int("RANK", 0)
    if rank != 0:
        return
    from oracle import ref
    if not ref.build():
        print(json.dumps({"impl": "reference",
                          "unavailable": "reference engine library oracle/_ref not built"}))
        return
    lib = ref.lib()
    threads = os.cpu_count() or 1
    # Rank 0's shard of the job's world list (the whole list at N=1).
    from maul3d_b200.shard import partition, shard_sizes, world_cost
    world_size = env_int("WORLD_SIZE", 1)
    all_sizes = shard_sizes(lib, args.seed, args.worlds * world_size, args.lo, args.hi)
    mine = partition([world_cost(n) for n in all_sizes], world_size)[0]
    sizes = [all_sizes[i] for i in mine]
    seeds = [args.seed + i for i in mine]

    def run_pool(worlds, order, steps) -> float:
        queue = list(order)
        lock = threading.Lock()

        def worker():
            while True:
                with lock:
                    if not queue:
                        return
                    k = queue.pop(0)
                lib.m3o_step_trace(worlds[k].id, DT, args.substeps, steps, None)

        t0 = time.perf_counter()
        pool = [threading.Thread(target=worker) for _ in range(min(threads, len(order)))]
        for t in pool:
            t.start()
        for t in pool:
            t.join()
        return time.perf_counter() - t0

    total_s = 0.0
    waves = 0
    for first in range(0, len(sizes), 64):
        wave = list(range(first, min(first + 64, len(sizes))))
        worlds = [ref.RefWorld.scene(SCENE_UNEVEN, seeds[i], sizes[i]) for i in wave]
        order = sorted(range(len(wave)), key=lambda k: -sizes[wave[k]])
        run_pool(worlds, order, args.warmup)
        total_s += run_pool(worlds, order, args.steps)
        for w in worlds:
            w.destroy()
        waves += 1
    total_bs = body_substeps(sizes, args.substeps, args.steps)
    value = total_bs / total_s
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference",
        "n_gpus": world_size, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * total_s / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": config_block(args, total_dynamic_bodies_per_gpu=int(sum(sizes))),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"all {len(sizes)} worlds in {waves} waves of <= 64 (the "
                                   f"reference's world table), {args.warmup} untimed + "
                                   f"{args.steps} timed steps each, {threads} host threads, "
                                   f"one world per task, largest first"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def terrain_run(m3, args, seed: int) -> dict:
    """Batched heightfield worlds: spheres, capsules and boxes settling on
    seeded terrain (the heightfield narrowphase), body counts log-uniform
    in [32, 512].  Device-resident steps timed with CUDA events; the
    reference steps a bounded sample of the same worlds on the host cores,
    and every sampled world's hash is compared with the device's."""
    import torch
    from oracle import ref
    count = args.terrain_worlds
    sizes = world_sizes(m3.lib, seed, count, 32, 512)
    batch = m3.WorldBatch([m3.World.scene(SCENE_TERRAIN, seed + i, n)
                           for i, n in enumerate(sizes)])
    m3.reserve_worlds(batch)
    m3.upload_worlds(batch)
    steps = args.terrain_steps
    m3.step_worlds(batch, DT, args.substeps, 3)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    m3.step_worlds(batch, DT, args.substeps, steps)
    m3.synchronize()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    value = body_substeps(sizes, args.substeps, steps) / (ms / 1000.0)
    got = m3.hash_worlds(batch)
    # Reference: the first worlds, each stepped the same 3 + `steps` steps.
    lib = ref.lib()
    threads = min(16, os.cpu_count() or 1)
    sample = []
    budget = max(2.0, args.cpu_seconds / 2)
    busy = 0.0
    mismatches = 0
    k = 0
    while k < count and busy < budget:
        wave = list(range(k, min(k + threads, count)))
        k = wave[-1] + 1
        worlds = [ref.RefWorld.scene(SCENE_TERRAIN, seed + i, sizes[i]) for i in wave]
        pool = [threading.Thread(target=lib.m3o_step_trace,
                                 args=(w.id, DT, args.substeps, 3 + steps, None)) for w in worlds]
        t0 = time.perf_counter()
        for t in pool:
            t.start()
        for t in pool:
            t.join()
        busy += time.perf_counter() - t0
        for i, w in zip(wave, worlds):
            mismatches += int(w.hash() != int(got[i]))
            w.destroy()
        sample.extend(wave)
    cpu = body_substeps([sizes[i] for i in sample], args.substeps, 3 + steps) / busy
    for w in batch:
        w.destroy()
    return {"workload": f"{count} heightfield worlds, bodies log-uniform [32, 512] "
                        "(spheres, capsules, boxes on seeded terrain)",
            "value": value, "unit": UNIT, "steps": steps, "ms_per_step": ms / steps,
            "cpu_reference": {"value": cpu, "unit": UNIT, "cores": threads,
                              "sample": f"first {len(sample)} worlds, {3 + steps} steps each"},
            "bit_exact_check": {"worlds_checked": len(sample), "mismatches": mismatches}}


SERVING_RATES = [100.0, 400.0, 1000.0, 4000.0, 20000.0, 0.0]
SERVING_CLIENTS = 4
# At most this many requests preparing or active: a tick steps every
# active request's frame, so the cap bounds a tick's time (and with it the
# latency of everything in flight); bursts wait in the queue.
SERVING_MAX_ACTIVE = 256


def reference_serving(containers, caps, threads: int) -> tuple[float, list[int]]:
    """The reference serving the same containers on the host cores: per
    request a fresh world of the snapshot's capacities, m3World_Restore,
    m3World_JournalReplay, m3World_Hash; requests in waves of 64 (its
    world table), worlds created serially, restore + replay one request
    per task on `threads` threads.  Returns (seconds, hashes)."""
    from oracle import ref
    lib = ref.abi.bind_replay(ref.abi.bind_snapshot(ref.abi.bind_create(ref.lib())))
    hashes = [0] * len(containers)
    t0 = time.perf_counter()
    for first in range(0, len(containers), 64):
        wave = list(range(first, min(first + 64, len(containers))))
        ids = {}
        for i in wave:
            d = lib.m3DefaultWorldDef()
            (d.bodyCapacity, d.shapeCapacity, d.meshCapacity, d.jointCapacity, d.voxelCapacity,
             d.characterCapacity) = caps[i]
            ids[i] = lib.m3CreateWorld(C.byref(d))
        queue = list(wave)
        lock = threading.Lock()
        failed = []

        def worker():
            while True:
                with lock:
                    if not queue:
                        return
                    i = queue.pop(0)
                snap, journal = containers[i]
                sb = (C.c_uint8 * len(snap)).from_buffer_copy(snap)
                jb = (C.c_uint8 * len(journal)).from_buffer_copy(journal)
                if not (lib.m3World_Restore(ids[i], sb, len(snap)) and
                        lib.m3World_JournalReplay(ids[i], jb, len(journal))):
                    failed.append(i)

        pool = [threading.Thread(target=worker) for _ in range(min(threads, len(wave)))]
        for t in pool:
            t.start()
        for t in pool:
            t.join()
        for i in wave:
            hashes[i] = 0 if i in failed else int(lib.m3World_Hash(ids[i]))
            lib.m3DestroyWorld(ids[i])
    return time.perf_counter() - t0, hashes


def serving_run(m3, distinct: int, seed: int, rates: list[float], budget: int,
                cpu_baseline: bool) -> dict:
    """Serving: replay containers of the served configuration's worlds
    (200-5000 bodies, log-uniform: boxes, spheres and 16-point QuickHull
    hulls on a plane, stepped 5 steps in) plus a journal of 4-16 frames,
    each 1-8 linear impulses of 1-50 N s on random bodies and one step of
    1/60 s in 4 substeps.  Requests arrive as a Poisson process at each
    rate (`distinct` different containers, submitted in turn from four
    client threads; per rate about one second of arrivals, 256-2048
    requests; rate 0 submits `distinct` at once); one server on this GPU
    under a device budget batches every active request's frame per tick
    on the main thread.  Latency is arrival to
    final hash.  An untimed warm-up serves every container once first.
    Every answer is compared with the reference's restore + replay of the
    same container, which is also timed on the host cores (all at once)
    as the serving baseline."""
    from maul3d_b200 import abi
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(200), np.log(5000), distinct)).astype(int)
    containers, raw, caps, work = [], [], [], []
    for i, n in enumerate(sizes):
        w = m3.World.scene(abi.SCENE_MIXED, seed + i, int(n))
        m3.step_worlds([w], DT, 4, 5)  # in motion, with contacts and warm starts
        bodies = w.body_count()
        frames = int(rng.integers(4, 17))
        journal = b""
        for _ in range(frames):
            for _ in range(int(rng.integers(1, 9))):
                d = rng.normal(size=3)
                d = d / np.linalg.norm(d) * rng.uniform(1.0, 50.0)
                journal += abi.journal_body_command(abi.OP_APPLY_LINEAR_IMPULSE,
                                                    int(rng.integers(2, bodies + 1)), 0,
                                                    [float(x) for x in d.astype(np.float32)])
            journal += abi.journal_step(DT, 4)
        snap = m3.snapshot(w)
        containers.append(abi.encode_container(m3.lib, snap, journal))
        raw.append((snap, journal))
        caps.append(tuple(int.from_bytes(snap[o:o + 4], "little")
                          for o in (24, 44, 92, 112, 132, 152)))
        work.append(int(n) * frames * 4)
        w.destroy()
    out = {"workload": f"{distinct} distinct containers: worlds of 200-5000 bodies "
                       "(log-uniform; boxes, spheres, 16-point hulls), 4-16 frames of 1-8 "
                       "impulses of 1-50 N s, 4 substeps",
           "device_budget_bytes": budget, "max_active": SERVING_MAX_ACTIVE,
           "clients": SERVING_CLIENTS, "runs": []}
    served = {}
    mismatched_runs = 0
    # Untimed warm-up: every distinct container once, all at once (a
    # long-running server's host and device memory pools are warm).
    warm = m3.Server(device_budget=budget, max_active=SERVING_MAX_ACTIVE)
    for c in containers:
        warm.submit(c)
    for ticket, (h, st) in warm.run().items():
        served[ticket - 1] = h if st == 0 else -st
    warm.close()
    for rate in rates:
        count = distinct if rate <= 0 else int(min(2048, max(256, rate)))
        arrivals = (np.cumsum(rng.exponential(1.0 / rate, count)) if rate > 0
                    else np.zeros(count))
        server = m3.Server(device_budget=budget, max_active=SERVING_MAX_ACTIVE)
        latency = np.zeros(count)
        finished = ticks = 0
        index_of = {}
        lock = threading.Lock()
        t0 = time.perf_counter()

        def client(part):
            # Arrivals part, part + CLIENTS, ...: submitted from their own
            # thread at their arrival times (the container copy happens in
            # the submitting thread, as a network thread's would).
            for i in range(part, count, SERVING_CLIENTS):
                delay = arrivals[i] - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
                ticket = server.submit(containers[i % distinct])
                with lock:
                    index_of[ticket] = i

        clients = [threading.Thread(target=client, args=(k,)) for k in range(SERVING_CLIENTS)]
        for c in clients:
            c.start()
        pending = []  # (ticket, done_at, answer) polled before the ticket was recorded
        while finished < count:
            if server.tick() == 0:
                time.sleep(0.0002)  # nothing queued or running
            ticks += 1
            t, h, st = server.poll()
            done_at = time.perf_counter() - t0
            pending.extend((int(t[k]), done_at, int(h[k]) if int(st[k]) == 0 else -int(st[k]))
                           for k in range(len(t)))
            with lock:
                resolved = [(index_of[tk], at, ans) for tk, at, ans in pending if tk in index_of]
                pending = [p for p in pending if p[0] not in index_of]
            for i, at, answer in resolved:
                latency[i] = at - arrivals[i]
                finished += 1
                if served.setdefault(i % distinct, answer) != answer:
                    mismatched_runs += 1
        wall = time.perf_counter() - t0
        for c in clients:
            c.join()
        stats = server.stats()
        server.close()
        out["runs"].append({
            "arrival_rate_per_s": rate if rate > 0 else "all at once",
            "requests": count,
            "p50_latency_ms": float(np.percentile(latency, 50) * 1e3),
            "p99_latency_ms": float(np.percentile(latency, 99) * 1e3),
            "requests_per_s": count / wall,
            "body_substeps_per_s": float(sum(work[i % distinct] for i in range(count))) / wall,
            "ticks": ticks, "peak_active": stats["peakActive"],
            "peak_device_bytes": stats["peakHeldBytes"],
            "host_ms": {k: round(stats[k], 1) for k in
                        ("prepareMs", "admitMs", "stepMs", "retireMs", "waitMs")},
            "workers": stats["workers"]})
    out["same_answer_every_time"] = mismatched_runs == 0
    if cpu_baseline:
        threads = os.cpu_count() or 1
        secs, ref_hashes = reference_serving(raw, caps, threads)
        mism = sum(1 for i in range(distinct) if served.get(i) != ref_hashes[i])
        out["cpu_reference"] = {
            "requests_per_s": distinct / secs,
            "body_substeps_per_s": float(sum(work)) / secs, "cores": threads,
            "kind": "reference",
            "sample": f"the {distinct} distinct containers at once: restore + journal replay "
                      f"+ hash per request, one request per task"}
        out["bit_exact_check"] = {"requests_checked": distinct, "mismatches": mism,
                                  "against": "the reference's restore + replay"}
    return out


# ---------------------------------------------------------------------------
# Single large worlds (the wide path: one world over the whole grid)
# ---------------------------------------------------------------------------
# (key, workload, scene, seed, param, substeps, device steps, window start,
#  reference window steps, reference build)
SINGLE_WORLDS = [
    ("c1", "box pyramid: a 20-row wall of 210 unit boxes on a plane (1000 steps)",
     1, 0, 20, 4, 1000, 0, 1000, "stock"),
    ("c2", "rain field: 10,000 spheres, capsules and QuickHull hulls falling 5-100 m onto a "
           "255 x 255 heightfield (600 steps)", 10, 3, 10000, 4, 600, 300, 10, "stock"),
    ("c5", "city: 1000 towers of 10 x 10 x 2 boxes welded by 460,000 breakable fixed joints, "
           "4000 projectiles, 8 substeps", 9, 5, 1000, 8, 13, 3, 1, "big"),
]


def _golden_hash(scene: int, seed: int, param: int, step: int):
    """The reference's hash after `step` steps from the committed traces
    (tests/golden), or None."""
    for name in ("large_traces.json", "traces.json"):
        path = ROOT / "tests" / "golden" / name
        if not path.exists():
            continue
        for c in json.loads(path.read_text())["cases"]:
            if (c["scene"], c["seed"], c["param"]) != (scene, seed, param):
                continue
            if "trace" in c and step <= len(c["trace"]):
                return c["trace"][step - 1]
            if "hashes" in c and str(step) in c["hashes"]:
                return c["hashes"][str(step)]
    return None


def single_world_run(m3, args, spec) -> dict:
    """One large world stepped alone: the device's body-substeps/s over
    the whole run (CUDA events, every stream idle at the end), the world
    hash checked against the reference's recorded trace; beside it the
    reference on the host cores, serially and on all host threads through
    its own task hooks, over a window of the same run (the device world's
    snapshot at the window's start, restored into the reference: same
    state, same steps), its hashes checked too."""
    import torch
    from oracle import ref
    key, workload, scene, seed, param, substeps, steps, start, window, variant = spec
    g = m3.World.scene(scene, seed, param)
    bodies = g.body_count() - 1  # the static ground body is not simulated
    m3.reserve_worlds([g])
    m3.upload_worlds([g])
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    ms = 0.0
    snap = None
    done = 0
    for chunk in ([start, steps - start] if start > 0 else [steps]):
        torch.cuda.synchronize()
        e0.record()
        m3.step_worlds([g], DT, substeps, chunk)
        m3.synchronize()
        e1.record()
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
        done += chunk
        if done == start:
            snap = m3.snapshot(g)
    got = f"{int(m3.hash_worlds([g])[0]):016x}"
    want = _golden_hash(scene, seed, param, steps)
    tc = time.perf_counter()
    m3.flush_trees([g])
    tree_ms = (time.perf_counter() - tc) * 1e3
    # The window's continuation from the restored snapshot, on the device
    # and in the reference, each compared with the reference's
    # uninterrupted run.  (On the rain field the reference's own restore
    # into a freshly built world does not reproduce its uninterrupted run:
    # its first step after such a restore depends on what earlier steps
    # left in its memory, not only on the snapshot; the device's restore
    # does reproduce it.)
    window_hash = None
    if snap is not None:
        gr = m3.World.scene(scene, seed, param)
        buf = (C.c_uint8 * len(snap)).from_buffer_copy(snap)
        if m3.lib.m3World_Restore(gr.id, buf, len(snap)):
            gr.step(DT, substeps, window)
            window_hash = gr.hash()
        gr.destroy()
    value = bodies * substeps * steps / (ms / 1000.0)
    line = {"workload": workload, "bodies": bodies, "substeps": substeps, "steps": steps,
            "value": value, "unit": UNIT, "ms_per_step": ms / steps,
            "tree_catchup_ms": tree_ms,
            "hash_check": {"step": steps, "device": got, "reference": want,
                           "equal": want is not None and got == want}}
    g.destroy()
    # The reference over the window [start, start + window).
    if args.no_cpu_baseline or not ref.build():
        return line
    lib = ref.lib(variant)
    threads = os.cpu_count() or 1
    out = {}
    for label, nthreads in (("serial", 1), ("threads", threads)):
        r = ref.RefWorld.scene(scene, seed, param, variant=variant)
        if snap is not None:
            ref.abi.bind_snapshot(lib)
            buf = (C.c_uint8 * len(snap)).from_buffer_copy(snap)
            if not lib.m3World_Restore(r.id, buf, len(snap)):
                r.destroy()
                line["cpu_reference"] = {"unavailable": "the reference refused the snapshot"}
                return line
        used = r.use_threads(nthreads)
        t0 = time.perf_counter()
        r.step(DT, substeps, window)
        sec = time.perf_counter() - t0
        h = r.hash()
        r.destroy()
        out[label] = {"value": bodies * substeps * window / sec, "unit": UNIT, "cores": used,
                      "ms_per_step": 1000.0 * sec / window}
        wantw = _golden_hash(scene, seed, param, start + window)
        out[label]["hash_equal"] = wantw is not None and f"{h:016x}" == wantw
    out["window"] = f"steps {start + 1}-{start + window} (the device world's snapshot after " \
                    f"step {start}, restored into the reference)" if start > 0 else \
                    f"steps 1-{window} from creation"
    out["kind"] = "reference" + (" (scratch cap raised: the stock build stalls)"
                                 if variant == "big" else "")
    if snap is not None:
        wantw = _golden_hash(scene, seed, param, start + window)
        out["device_restored_equal"] = (window_hash is not None and wantw is not None and
                                        f"{window_hash:016x}" == wantw)
    line["cpu_reference"] = out
    return line


def config_block(args, **extra) -> dict:
    cfg = {"workload": f"batched uneven worlds: {args.worlds} worlds per GPU, dynamic bodies "
                       f"log-uniform [{args.lo}, {args.hi}], box stacks + spheres + 3 revolute "
                       f"capsule chains, dt 1/60, {args.substeps} substeps",
           "worlds_per_gpu": args.worlds, "substeps": args.substeps, "dt": DT, "seed": args.seed,
           "l2": "inputs larger than L2 (world slabs total several GB)",
           "parallelism": "one block per world; worlds split across ranks by estimated cost, "
                          "bodies + pairs (weak scaling)"}
    cfg.update(extra)
    return cfg


# ---------------------------------------------------------------------------
# Device arm
# ---------------------------------------------------------------------------
def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--tune-steps", type=int, default=24,
                    help="untimed steps of the packing autotuner, on a copy of the batch (0: none)")
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--worlds", type=int, default=4096)
    ap.add_argument("--lo", type=int, default=32)
    ap.add_argument("--hi", type=int, default=2048)
    ap.add_argument("--substeps", type=int, default=4)
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--plain-sample", type=int, default=64)
    ap.add_argument("--ref-sample", type=int, default=64)
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--serving-requests", type=int, default=256,
                    help="distinct serving containers (0: no serving run)")
    ap.add_argument("--serving-budget-gb", type=int, default=16,
                    help="the server's device memory budget")
    ap.add_argument("--serving-only", action="store_true",
                    help="run only the serving sweep, print it and exit")
    ap.add_argument("--terrain-worlds", type=int, default=1024)
    ap.add_argument("--terrain-steps", type=int, default=20)
    ap.add_argument("--single", default="c1,c2,c5",
                    help="single large worlds to run after the batch (comma list, or none)")
    ap.add_argument("--single-only", action="store_true",
                    help="run only the single large worlds (profiling), print them and exit")
    ap.add_argument("--city-towers", type=int, default=1000,
                    help="towers of the c5 city world (1000 in the configuration)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    if args.impl == "reference":
        run_reference_arm(args)
        return

    import torch
    import torch.distributed as dist
    import maul3d_b200 as m3

    rank = env_int("RANK", 0)
    world_size = env_int("WORLD_SIZE", 1)
    local_rank = env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local_rank)
    m3.set_device(local_rank)
    if args.serving_only:
        print(json.dumps({"serving": serving_run(m3, args.serving_requests, args.seed + 77,
                                                 SERVING_RATES, args.serving_budget_gb << 30,
                                                 not args.no_cpu_baseline)}))
        return
    if args.single_only:
        want = set(args.single.split(","))
        specs = [spec for spec in SINGLE_WORLDS if spec[0] in want]
        specs = [spec[:4] + (args.city_towers,) + spec[5:] if spec[0] == "c5" else spec
                 for spec in specs]
        print(json.dumps({spec[0]: single_world_run(m3, args, spec) for spec in specs}))
        return
    if world_size > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))

    # Weak scaling: the job's world list holds `worlds` per GPU; every
    # rank computes the same cost-balanced split of it and builds only its
    # own shard (at N=1 the shard is the whole list, in order).
    from maul3d_b200.shard import partition, shard_sizes, world_cost
    all_sizes = shard_sizes(m3.lib, args.seed, args.worlds * world_size, args.lo, args.hi)
    mine = partition([world_cost(n) for n in all_sizes], world_size)[rank]
    sizes = [all_sizes[i] for i in mine]
    seeds = [args.seed + i for i in mine]
    rank_seed = args.seed + 1_000_003 * rank
    # The packing autotuner, on a batch of the same worlds built apart (its
    # steps are real steps; the timed batch then starts from creation).
    packing = m3.get_packing()
    packing_ms = None
    trials = []
    if args.tune_steps > 0:
        tune = m3.WorldBatch(build_worlds(m3, sizes, seeds))
        m3.reserve_worlds(tune)
        m3.upload_worlds(tune)
        packing, packing_ms = m3.autotune_packing(tune, DT, args.substeps, args.tune_steps)
        trials = m3.autotune_trials()
        for w in tune:
            w.destroy()
    worlds = m3.WorldBatch(build_worlds(m3, sizes, seeds))
    m3.reserve_worlds(worlds)
    m3.upload_worlds(worlds)

    # Warm-up steps (untimed), and their tree moves replayed: the timed
    # steps' catch-up is reported apart, below.
    m3.step_worlds(worlds, DT, args.substeps, args.warmup)
    m3.flush_trees(worlds)
    stats0 = np.stack([m3.world_stats(w) for w in worlds])

    sampler = ClockSampler(local_rank)
    sampler.start()
    if world_size > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    launches0 = m3.launch_count()
    e0.record()
    m3.step_worlds(worlds, DT, args.substeps, args.steps)
    # The trees finish on their own stream behind the call: the timed
    # region ends when every stream of the device is idle.
    m3.synchronize()
    e1.record()
    launches = m3.launch_count() - launches0
    torch.cuda.synchronize()
    if world_size > 1:
        dist.barrier()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    stage_ms = m3.kernel_ms()
    # The broadphase trees are snapshot state, replayed from the recorded
    # leaf moves when read (or every 16 steps): the catch-up of whatever
    # the timed steps left unreplayed, timed on its own.
    t0 = time.perf_counter()
    m3.flush_trees(worlds)
    tree_catchup_ms = (time.perf_counter() - t0) * 1e3
    stats1 = np.stack([m3.world_stats(w) for w in worlds])
    work = (stats1 - stats0).astype(np.float64).sum(axis=0)
    # The device hash of the whole batch, timed alone on the device.
    h0 = torch.cuda.Event(enable_timing=True)
    h1 = torch.cuda.Event(enable_timing=True)
    h0.record()
    device_hashes = m3.hash_worlds(worlds).copy()
    h1.record()
    torch.cuda.synchronize()
    hash_ms = h0.elapsed_time(h1)

    local_bs = body_substeps(sizes, args.substeps, args.steps)
    if world_size > 1:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
        b = torch.tensor([float(local_bs)], dtype=torch.float64, device="cuda")
        dist.all_reduce(b, op=dist.ReduceOp.SUM)
        total_bs = float(b.item())
    else:
        ms_max = ms
        total_bs = float(local_bs)
    value = total_bs / (ms_max / 1000.0)

    # Roofline of the dominant kernel (m3SubstepKernel, the substep loop:
    # integrate, warm start, solve, relax, restitution, store):
    # algorithmic bytes of its per-substep row and body passes / its
    # device time from CUDA events around it on the launching stream.
    sub_bytes = (BYTES_PER_MOVER_SUBSTEP * work[0] + BYTES_PER_CONTACT_SUBSTEP * work[1] +
                 BYTES_PER_JOINT_SUBSTEP * work[2])
    peak, peak_kind = measured_peaks()
    kms = stage_ms["substep"]
    achieved = (sub_bytes / args.steps) / (kms / args.steps / 1000.0) / 1e9
    roofline = {"kernel": "m3SubstepKernel", "bound": "hbm", "achieved": achieved,
                "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                "limiter": "latency: dependent row solves between block barriers; rows and "
                           "bodies are re-read from L1, L2 and shared memory, so DRAM traffic "
                           "stays below the algorithmic bytes",
                "traffic": SUBSTEP_TRAFFIC_DEFAULT if default_workload(args) else None,
                "traffic_source": "ncu dram bytes of one step's three size-class launches on "
                                  "this workload",
                "bytes_per_launch": sub_bytes / args.steps,
                "launch_ms": kms / args.steps,
                "share": {k: v / ms for k, v in stage_ms.items()}}

    # Plain path: one world per launch sequence, a sample of the worlds.
    plain = None
    if rank == 0 and args.plain_sample > 0:
        psizes = sizes[:args.plain_sample]
        pworlds = build_worlds(m3, psizes, seeds[:len(psizes)])
        m3.reserve_worlds(pworlds)
        m3.upload_worlds(pworlds)
        for w in pworlds:
            w.step(DT, args.substeps, 1)
        torch.cuda.synchronize()
        p0 = torch.cuda.Event(enable_timing=True)
        p1 = torch.cuda.Event(enable_timing=True)
        device_ms = 0.0
        p0.record()
        for _ in range(args.steps):
            for w in pworlds:
                m3.step_worlds([w], DT, args.substeps, 1)
                device_ms += m3.profile(w)["step"]
        m3.synchronize()
        p1.record()
        torch.cuda.synchronize()
        pms = p0.elapsed_time(p1)
        calls = args.steps * len(pworlds)
        plain = {"value": body_substeps(psizes, args.substeps, args.steps) / (pms / 1000.0),
                 "unit": UNIT, "sample_worlds": len(psizes),
                 "ms_per_call": pms / calls,
                 "device_stage_ms_per_call": device_ms / calls,
                 "note": "each world stepped by its own launch sequence; device_stage_ms is "
                         "the sum of the five stages' event times of each call"}
        for w in pworlds:
            w.destroy()

    # End to end through the C ABI: fresh host-built worlds, their upload,
    # K steps and a D2H hash read of every world after every step.
    e2e = None
    if not args.no_e2e:
        eworlds = m3.WorldBatch(build_worlds(m3, sizes, seeds))
        tr = time.perf_counter()
        m3.reserve_worlds(eworlds)
        reserve_ms = (time.perf_counter() - tr) * 1e3
        up0 = m3.uploaded_bytes()
        if world_size > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        m3.upload_worlds(eworlds)
        t1 = time.perf_counter()
        h2d = m3.uploaded_bytes() - up0
        step_s = 0.0
        hash_s = 0.0
        for _ in range(args.steps):
            ta = time.perf_counter()
            m3.step_worlds(eworlds, DT, args.substeps, 1)
            tb = time.perf_counter()
            m3.hash_worlds(eworlds)
            step_s += tb - ta
            hash_s += time.perf_counter() - tb
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t0
        if world_size > 1:
            t = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        e2e = {"value": total_bs / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": int(h2d // args.steps),
               "d2h_bytes_per_step": 8 * len(eworlds),
               "reserve_ms_untimed": reserve_ms,
               "upload_ms": (t1 - t0) * 1e3,
               "step_ms_per_step": step_s * 1e3 / args.steps,
               "hash_ms_per_step": hash_s * 1e3 / args.steps,
               "note": "world images uploaded once inside the timed region (page-locked host "
                       "memory); per step: batched step + device hash of every world read back"}
        for w in eworlds:
            w.destroy()

    # CPU baseline: the reference engine on the host cores, same worlds,
    # same W+K steps; every sampled world's final hash must equal the
    # device's (the bit-exact check behind the metric's name).
    cpu = None
    verified = None
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        from oracle import ref
        if ref.build():
            threads = os.cpu_count() or 1
            bs, busy, hashes, n = reference_run(sizes, args.seed, args.substeps,
                                                args.warmup + args.steps, threads,
                                                args.cpu_seconds, want_hashes=True)
            mismatched = [i for i, h in hashes.items() if int(device_hashes[i]) != h]
            verified = {"worlds_checked": len(hashes), "mismatches": len(mismatched)}
            cpu = {"value": bs / busy, "unit": UNIT, "cores": threads, "kind": "reference",
                   "sample": f"first {n} of {len(sizes)} worlds (waves of <= 64), "
                             f"{args.warmup + args.steps} steps each, {threads} host threads; "
                             f"every sampled world's final hash compared with the device's"}

    serving = None
    if args.serving_requests > 0 and rank == 0:
        serving = serving_run(m3, args.serving_requests, rank_seed + 77, SERVING_RATES,
                              args.serving_budget_gb << 30, not args.no_cpu_baseline)
    # The terrain batch runs after the serving loop, so that its host
    # threads and device memory leave the latency figures alone.
    singles = None
    if rank == 0 and args.single not in ("", "none"):
        want = set(args.single.split(","))
        singles = {spec[0]: single_world_run(m3, args, spec) for spec in SINGLE_WORLDS
                   if spec[0] in want}
    terrain = None
    if rank == 0 and args.terrain_worlds > 0 and not args.no_cpu_baseline:
        terrain = terrain_run(m3, args, rank_seed + 91)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world_size,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64", "data": "synthetic",
            "config": config_block(args, total_dynamic_bodies_per_gpu=int(sum(sizes))),
            "e2e": e2e, "gpu_launches": launches, "roofline": roofline,
            "cpu_baseline": cpu, "plain_gpu": plain, "bit_exact_check": verified,
            "hash_ms": hash_ms, "clocks": clocks, "terrain": terrain, "serving": serving,
            "single_worlds": singles,
            "packing": {"note": "the batch's packing onto the SMs (size-class bounds in shape "
                                "slots, threads per world, shared-memory budget per class) "
                                "chosen by the autotuner on a copy of the batch (same worlds, "
                                "its own untimed steps from creation); trials: each candidate's "
                                "prepare + substep ms against the mean of the steps beside it",
                        "tune_steps": args.tune_steps, "chosen": packing,
                        "prepare_substep_ms_per_step": packing_ms,
                        "trials": [{"packing": t["packing"], "ms": round(t["ms"], 3),
                                    "baseline_ms": round(t["baseline_ms"], 3),
                                    "adopted": t["adopted"]} for t in trials]},
            "tree": {"note": "the broadphase tree (snapshot state) replays recorded leaf moves "
                             "every 16 steps beside the steps, or when read; catchup_ms = "
                             "replaying what the timed steps left, after them",
                     "catchup_ms": tree_catchup_ms,
                     "value_with_catchup": total_bs / ((ms_max + tree_catchup_ms) / 1000.0)},
        }
        print(json.dumps(line))
    if world_size > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
