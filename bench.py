#!/usr/bin/env python
"""Body-substeps/s of the GPU world on the streaming mixed-rain workload.

Workload (one "step"): the 20,000-body streaming mixed rain (spheres,
capsules and boxes in thirds over a 100x60x100 m volume, seeded synthetic
data) advanced by one m3d_world_step at 60 Hz with 4 substeps, after the 200
lowest dynamic bodies are destroyed and 200 new ones spawned through the C
API.  Both arms first run --preroll untimed steps (300 by default), so the
timed window is the settled rain (piles on the ground, churn removing the
lowest bodies) rather than the initial free fall, then --warmup untimed
steps.  Metric: body-substeps/s = dynamic bodies x substeps per step, summed
over the timed steps, divided by the time.

  value  device time of the steps: CUDA events on the world's stream around
         each m3d_world_step (uploads of the step's new bodies included);
  e2e    host wall time of the same steps through the C ABI, churn included:
         the H2D copies of the spawned bodies, the D2H pose read used to pick
         the lowest bodies and the per-step event/counter reads.
The L2 (126 MB) is flushed between timed steps by a 256 MiB write.

--impl reference times the reference's own CPU implementation (the
reference library built from its sources with its release flags) on the
same workload, pre-roll and window with all host threads.  N > 1 (torchrun)
runs one independent replica of the rain per GPU (a single world does not
shard); value is the sum of the replicas' work over the slowest replica's
time.  At N > 1 the line also carries the batched-worlds workload sharded by
world across the ranks (variants.batched_sharded).

The line's `variants` (N = 1) carry the batched-worlds, settled-pile and
forward+adjoint workloads, each with its own roofline object and CPU sample.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import ctypes as C

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from melon3d_b200 import api, harness  # noqa: E402

WORKLOAD = "streaming mixed rain, 20000 bodies, churn 200/step, 60 Hz x 4 substeps"
REF_RELEASE_LIB = os.path.join(ROOT, "oracle", "_ref", "libmelon3d_ref_fast.so")
COUNTER_NAMES = ["activeEntries", "stableEntries", "activeOversized", "stableOversized", "runs", "gridPairs",
                 "overPairs", "newContacts", "removed", "endRemoval", "beginNP", "endNP", "anyAwakeDynamic",
                 "islandCount", "touchingCount", "awakeIslands", "islandContacts", "islandJoints", "islandBodies",
                 "stableDirty", "bodyCount", "awakeBodyCount", "hashFail", "coloredIslands", "serialIslands",
                 "freeIslands", "waitErrors", "contactCount", "giantIslands", "keptStable", "keptStableOver",
                 "keptContacts", "tinyIslands", "warpIslands", "islandPoints", "serialBodies", "serialContacts"]


def _serial_bytes(c, sub):
    # per substep 300 B per body (integrate 220 + reconstruct 80), 320 B per
    # manifold point and 884 B per contact (prepare, two normal iterations,
    # friction, velocity pass), the serial islands' share of the points
    # taken in proportion to their contacts
    pts = c["islandPoints"] * c["serialContacts"] / max(c["islandContacts"], 1)
    return sub * (300.0 * c["serialBodies"] + 884.0 * c["serialContacts"] + 320.0 * pts)


def _coloured_bytes(c, sub):
    # the same per-substep figures for the bodies and contacts of the
    # coloured islands (all islands minus the serial and the single-body ones)
    bodies = max(c["islandBodies"] - c["serialBodies"] - c["freeIslands"], 0)
    contacts = max(c["islandContacts"] - c["serialContacts"], 0)
    pts = c["islandPoints"] * contacts / max(c["islandContacts"], 1)
    return sub * (300.0 * bodies + 884.0 * contacts + 320.0 * pts)


# A free body's fused substep loop keeps the body in registers: per step it
# reads pose, velocities, mass properties and 16 B of the cold record (96 B)
# and writes pose, velocities, their pre-substep copies and the world inverse
# inertia (176 B), whatever the substep count.
FREE_BODY_BYTES = 272.0

# Algorithmic bytes per step of the kernels reported against the roofline:
# each field a kernel must read or write, counted once (fp32 SoA).
ROOFLINE_MODELS = {
    # serial islands: the whole substep loop of every serial island
    "kSolveSerial": ("HBM bytes per serial-island body, contact and point per substep", _serial_bytes),
    "kSolveTiny": ("HBM bytes per serial-island body, contact and point per substep", _serial_bytes),
    # coloured islands solved on the whole GPU (the settled pile)
    "kSolveGiant": ("HBM bytes per coloured-island body, contact and point per substep", _coloured_bytes),
    # free-body islands: read once, written once per step
    "kSolveFree": ("HBM bytes per free body per step (272 B)", lambda c, sub: c["freeIslands"] * FREE_BODY_BYTES),
    # narrowphase: per live contact the two body indices, flags, two poses,
    # two cached poses, point count (~150 B); regenerated pairs also write
    # their manifold (~4 x 132 B) - counted as the cached case (a floor)
    "kNarrowphase": ("HBM bytes per contact", lambda c, sub: c["contactCount"] * 150.0),
}


def bench_config(args, world_size):
    """The `config` object of both arms' JSON lines (identical by design)."""
    return {"workload": WORKLOAD, "variant": "plain", "bodies": args.bodies, "churn_per_step": args.churn,
            "substeps": args.substeps, "hz": 60, "preroll_steps": args.preroll,
            "timed_window": "steps %d-%d (after %d untimed pre-roll and %d warm-up steps)" % (
                args.preroll + args.warmup, args.preroll + args.warmup + args.steps - 1, args.preroll, args.warmup),
            "l2": "flushed between timed steps (256 MiB write); CPU arm: not applicable",
            "parallelism": "replicas" if world_size > 1 else "single world"}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=120)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--preroll", type=int, default=300,
                   help="untimed steps run before the warm-up in both arms, so the timed window is the "
                        "settled rain (piles on the ground) rather than the initial free fall")
    p.add_argument("--impl", choices=["gpu", "reference"], default="gpu")
    p.add_argument("--bodies", type=int, default=20000)
    p.add_argument("--churn", type=int, default=200)
    p.add_argument("--substeps", type=int, default=4)
    p.add_argument("--roofline-kernels", default="kSolveSerial,kSolveFree,kNarrowphase,kSolveTiny")
    p.add_argument("--cpu-baseline-seconds", type=float, default=15.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-variants", action="store_true",
                   help="skip the batched-worlds and large-pile measurements")
    p.add_argument("--batch-worlds", type=int, default=4096)
    p.add_argument("--batch-steps", type=int, default=40)
    p.add_argument("--batch-solo-worlds", type=int, default=128,
                   help="worlds of the batch stepped one at a time through the plain path for the comparison")
    p.add_argument("--no-autotune", action="store_true", help="batch variant with the default kernel choice")
    p.add_argument("--pile-steps", type=int, default=12)
    p.add_argument("--pile-cpu-steps", type=int, default=20)
    p.add_argument("--adjoint-worlds", type=int, default=1024)
    p.add_argument("--adjoint-steps", type=int, default=120)
    p.add_argument("--only-adjoint", action="store_true",
                   help="run only the forward+adjoint measurement and print its JSON object")
    return p.parse_args()


class Dist:
    def __init__(self, n):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime
            import torch
            import torch.distributed as dist
            torch.cuda.set_device(self.local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", self.local))
            self.pg = dist

    def barrier(self):
        if self.pg is not None:
            self.pg.barrier()

    def reduce(self, value, op):
        if self.pg is None:
            return value
        import torch
        t = torch.tensor([float(value)], dtype=torch.float64, device="cuda")
        self.pg.all_reduce(t, op=getattr(self.pg.ReduceOp, op))
        return float(t.item())

    def close(self):
        if self.pg is not None:
            self.pg.destroy_process_group()


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""

    FIELDS = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"

    def __init__(self, gpu_index):
        self.proc = None
        self.index = gpu_index

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = max(mx, float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def read_traffic():
    """DRAM bytes per launch (read + write) of kernels captured with ncu on
    this workload, from profiles/dram_traffic.txt ("<kernel> <bytes>" lines);
    empty when the file is absent."""
    out = {}
    try:
        for line in open(os.path.join(ROOT, "profiles", "dram_traffic.txt")):
            parts = line.split()
            if len(parts) >= 2 and not line.startswith("#"):
                out[parts[0]] = float(parts[1])
    except OSError:
        pass
    return out


def flush_l2(buf):
    buf.fill_(1.0)


def run_reference_sample(steps, warmup, args, seconds_cap=None):
    """The reference's CPU step on the same workload (same seed, pre-roll
    and warm-up), all host threads."""
    if not os.path.exists(REF_RELEASE_LIB):
        return None, "oracle/_ref/libmelon3d_ref_fast.so not built"
    lib = api.bind(C.CDLL(REF_RELEASE_LIB))
    cores = os.cpu_count() or 1
    sc = harness.Scene(lib, harness.RAIN, 2, args.bodies, args.churn, 0, workers=cores)
    sc.run(args.preroll + warmup, args.substeps)
    done, bs_total, wall_total = 0, 0, 0.0
    while done < steps:
        bs, wall, _ = sc.run(1, args.substeps)
        bs_total += bs
        wall_total += wall
        done += 1
        if seconds_cap is not None and wall_total > seconds_cap * 1000.0:
            break
    sc.close()
    return {"value": bs_total / (wall_total / 1000.0), "unit": "body-substeps/s", "cores": cores,
            "kind": "reference",
            "sample": "%d steps (after %d pre-roll and %d warm-up steps) of the same workload, reference release "
                      "build, workerCount=%d" % (done, args.preroll, warmup, cores),
            "ms_per_step": wall_total / max(done, 1)}, None


def _peaks():
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        peaks = {}
    return float(peaks.get("hbm_gbs", 6650.0)), ("measured" if "hbm_gbs" in peaks else "fallback")


def _counters(lib, world):
    buf = (C.c_uint32 * 64)()
    n = lib.m3d_gpu_step_counters(world, buf, 64)
    return {name: buf[i] for i, name in enumerate(COUNTER_NAMES[:n])}


def _profiler_table(lib):
    table = C.create_string_buffer(1 << 16)
    lib.m3d_gpu_profiler_table(table, 1 << 16)
    out = {}
    for row in table.value.decode().splitlines():
        kname, kl, kms = row.split()
        out[kname] = (int(kl), float(kms))
    return out


class Timed:
    """Steps of one world through the C API with the model kernels bracketed
    by CUDA events: device time, wall time, the algorithmic bytes of each
    model kernel (from the step counters) and its event-timed duration."""

    def __init__(self, lib, world, kernels, substeps):
        self.lib, self.world, self.substeps = lib, world, substeps
        self.names = [k for k in kernels if k in ROOFLINE_MODELS]
        self.dev = self.wall = 0.0
        self.steps = 0
        self.bytes = {k: 0.0 for k in self.names}
        lib.m3d_gpu_profiler_reset(",".join(self.names).encode())

    def step(self, fn):
        t = time.perf_counter()
        fn()
        self.wall += (time.perf_counter() - t) * 1000.0
        self.dev += self.lib.m3d_gpu_last_step_device_ms(self.world)
        self.steps += 1
        c = _counters(self.lib, self.world)
        for k in self.names:
            self.bytes[k] += ROOFLINE_MODELS[k][1](c, self.substeps)

    def rooflines(self):
        """Roofline objects of the model kernels, dominant (largest share of
        the device time) first."""
        peak, source = _peaks()
        timed = _profiler_table(self.lib)
        traffic = read_traffic()
        roofs = []
        for k in self.names:
            if k not in timed or timed[k][0] == 0:
                continue
            kl, kms = timed[k]
            avg_s = kms / 1000.0 / kl
            per_launch = self.bytes[k] / kl
            achieved = per_launch / avg_s / 1e9
            roofs.append({"bound": "hbm", "kernel": k, "achieved": achieved, "peak": peak, "unit": "GB/s",
                          "frac": achieved / peak, "traffic": traffic.get(k), "bytes_per_launch": per_launch,
                          "avg_launch_us": avg_s * 1e6, "launches": kl, "share_of_step": kms / max(self.dev, 1e-9),
                          "model": ROOFLINE_MODELS[k][0], "peak_source": source + " (burst copy bandwidth)"})
        roofs.sort(key=lambda r: -r["share_of_step"])
        return roofs


def measure_pile(lib, args, ref_lib):
    """250,000-box settled pile (50x100x50 lattice), one giant island: the
    whole-GPU coloured solve.  Steps 0-1 (3.1M contacts created) untimed."""
    sc = harness.Scene(lib, harness.PILE, 3, 50, 100, 50)
    n = sc.sl.scn_dynamic_count(sc.handle)
    sc.run(2, args.substeps)
    tm = Timed(lib, sc.world, ["kSolveGiant", "kNarrowphase"], args.substeps)
    for _ in range(args.pile_steps):
        tm.step(lambda: lib.m3d_world_step(sc.world, 1.0 / 60.0, args.substeps))
    roofs = tm.rooflines()
    pr = lib.m3d_world_profile(sc.world)
    gp = (C.c_double * 15)()
    stages = None
    if lib.m3d_gpu_giant_profile(sc.world, gp, 15) == 15:
        stages = {"incidence_ms": gp[0] / 1e6, "colouring_ms": gp[1] / 1e6, "buckets_ms": gp[2] / 1e6,
                  "overflow_levels_ms": gp[3] / 1e6, "substeps_ms": gp[4] / 1e6, "colours": int(gp[5]),
                  "overflow_contacts": int(gp[6]), "overflow_levels": int(gp[7]),
                  "substep_stages_ms": {"integrate_prepare": gp[8] / 1e6, "coloured_normals": gp[9] / 1e6,
                                        "overflow_normals": gp[10] / 1e6, "friction": gp[11] / 1e6,
                                        "reconstruct": gp[12] / 1e6, "coloured_velocity": gp[13] / 1e6,
                                        "overflow_velocity": gp[14] / 1e6}}
    work = n * args.substeps * tm.steps
    out = {"workload": "settled pile, 250,000 boxes (50x100x50 lattice, 1.02 m spacing, jitter), one giant island",
           "bodies": n, "steps": tm.steps, "timed_window": "steps 2-%d" % (1 + tm.steps),
           "value": work / (tm.dev / 1000.0), "unit": "body-substeps/s", "ms_per_step": tm.dev / tm.steps,
           "e2e": {"value": work / (tm.wall / 1000.0), "ms_per_step": tm.wall / tm.steps},
           "roofline": roofs[0] if roofs else None, "roofline_others": roofs[1:], "giant_stages_last_step": stages,
           "contacts": pr.contactCount, "touching": pr.touchingContactCount, "status": lib.m3d_gpu_status(sc.world)}
    sc.close()
    if ref_lib is not None and not args.no_cpu_baseline:
        cores = os.cpu_count() or 1
        rs = harness.Scene(ref_lib, harness.PILE, 3, 50, 100, 50, workers=cores)
        rs.run(2, args.substeps)  # contact creation, as on the GPU
        bs, wall_ms, _ = rs.run(args.pile_cpu_steps, args.substeps)
        rs.close()
        out["cpu_baseline"] = {"value": bs / (wall_ms / 1000.0), "unit": "body-substeps/s", "cores": cores,
                               "kind": "reference",
                               "sample": "%d awake steps (steps 2-%d, measured, not extrapolated), reference "
                                         "release build, workerCount=%d" % (args.pile_cpu_steps,
                                                                             1 + args.pile_cpu_steps, cores)}
    return out


def _batch_from(lib, seeds):
    scenes = [harness.Scene(lib, harness.BATCH_WORLD, k) for k in seeds]
    bodies = [s.sl.scn_dynamic_count(s.handle) for s in scenes]
    arr = (C.c_void_p * len(scenes))(*[s.world for s in scenes])
    batch = lib.m3d_gpu_batch_create(arr, len(scenes)) if scenes else None
    return scenes, bodies, batch


def _world_centroids(lib, batch, count):
    """Centroid of each world's dynamic bodies after the last step."""
    n = lib.m3d_gpu_body_capacity(batch)
    pos = (C.c_float * (3 * max(n, 1)))()
    lib.m3d_gpu_read_poses(batch, pos, None, n)
    p = np.frombuffer(pos, dtype=np.float32).reshape(-1, 3)[:n].astype(np.float64)
    out = np.zeros((count, 3))
    for k in range(count):
        f0, f1 = lib.m3d_gpu_batch_first_body(batch, k), lib.m3d_gpu_batch_first_body(batch, k + 1)
        out[k] = p[f0 + 1:f1].mean(axis=0) if f1 > f0 + 1 else 0.0  # slot f0 is the world's ground box
    return out


BATCH_KERNELS = ["kSolveTiny", "kSolveSerial", "kNarrowphase", "kSolveFree"]


def measure_batch(lib, args, ref_lib):
    """4096 independent worlds (own ground, 16-512 bodies, 0-4 joints) in one
    batch, against the same worlds stepped one at a time through the plain
    path over the same window of steps."""
    W = args.batch_worlds
    scenes, counts, batch = _batch_from(lib, range(W))
    bodies = int(sum(counts))
    # one at a time: a sample of the same worlds through the plain path, the
    # same window (step 0 untimed, then batch_steps steps), device and wall
    solo_n = min(args.batch_solo_worlds, W)
    solo_dev = solo_wall = 0.0
    solo_bs = 0
    for s, cnt in zip(scenes[:solo_n], counts[:solo_n]):
        s.step_only(args.substeps)
        for _ in range(args.batch_steps):
            t = time.perf_counter()
            s.step_only(args.substeps)
            solo_wall += (time.perf_counter() - t) * 1000.0
            solo_dev += lib.m3d_gpu_last_step_device_ms(s.world)
            solo_bs += cnt * args.substeps
    for s in scenes:
        s.close()
    tuning = None
    if not args.no_autotune:
        # trials on a twin batch (steps 1-24), then this batch takes the
        # choice from the cache file at once; results do not depend on it
        import tempfile
        os.environ.setdefault("M3D_AUTOTUNE_CACHE", os.path.join(tempfile.gettempdir(), "m3d_autotune.txt"))
        if lib.m3d_gpu_autotune(batch, 2) == 0:
            twin_scenes, _, twin = _batch_from(lib, range(W))
            for s in twin_scenes:
                s.close()
            lib.m3d_gpu_autotune(twin, 2)
            while lib.m3d_gpu_autotune_state(twin, None, None) == 1:
                lib.m3d_world_step(twin, 1.0 / 60.0, args.substeps)
            lib.m3d_world_destroy(twin)
            lib.m3d_gpu_autotune(batch, 2)
        tc, tmi = C.c_int32(), C.c_int32()
        lib.m3d_gpu_autotune_state(batch, C.byref(tc), C.byref(tmi))
        tuning = {"tiny_island_contacts": tc.value, "tiny_mode_islands": tmi.value,
                  "cache": os.environ["M3D_AUTOTUNE_CACHE"]}
    lib.m3d_world_step(batch, 1.0 / 60.0, args.substeps)
    tm = Timed(lib, batch, BATCH_KERNELS, args.substeps)  # resets the launch counter
    launches0 = lib.m3d_gpu_profiler_launches()
    for _ in range(args.batch_steps):
        tm.step(lambda: lib.m3d_world_step(batch, 1.0 / 60.0, args.substeps))
    launches = lib.m3d_gpu_profiler_launches() - launches0
    roofs = tm.rooflines()
    work = bodies * args.substeps * tm.steps
    value, e2e = work / (tm.dev / 1000.0), work / (tm.wall / 1000.0)
    solo = {"value": solo_bs / (solo_dev / 1000.0), "e2e": solo_bs / (solo_wall / 1000.0), "unit": "body-substeps/s",
            "sample": "the first %d of the same worlds, each stepped alone through the plain GPU path over the same "
                      "window (steps 1-%d)" % (solo_n, args.batch_steps)}
    out = {"workload": "%d worlds, log-uniform 16-512 bodies each (rain shapes, own ground box, 0-4 ball/hinge "
                       "joints)" % W, "bodies": bodies, "steps": tm.steps,
           "timed_window": "steps 1-%d" % tm.steps, "value": value, "unit": "body-substeps/s",
           "ms_per_step": tm.dev / tm.steps, "e2e": {"value": e2e, "ms_per_step": tm.wall / tm.steps},
           "one_at_a_time": solo, "speedup_vs_one_at_a_time": {"device": value / solo["value"], "e2e": e2e / solo["e2e"]},
           "gpu_launches_per_step": launches / tm.steps, "autotuned": tuning, "roofline": roofs[0] if roofs else None,
           "roofline_others": roofs[1:], "status": lib.m3d_gpu_status(batch)}
    lib.m3d_world_destroy(batch)
    if ref_lib is not None and not args.no_cpu_baseline:
        cores = os.cpu_count() or 1
        rn, rsteps = min(256, W), 5
        wall = 0.0
        rbs = 0
        for k in range(rn):
            rs = harness.Scene(ref_lib, harness.BATCH_WORLD, k, workers=cores)
            rs.step_only(args.substeps)
            bs, w_ms, _ = rs.run(rsteps, args.substeps)
            rbs += bs
            wall += w_ms
            rs.close()
        out["cpu_baseline"] = {"value": rbs / (wall / 1000.0), "unit": "body-substeps/s", "cores": cores,
                               "kind": "reference", "sample": "%d worlds x steps 1-%d one after another, "
                                                              "workerCount=%d" % (rn, rsteps, cores)}
    return out


def measure_batch_sharded(lib, args, d):
    """The batched-worlds workload split by world across the ranks (greedy
    prefix split of the cumulative body count), each rank stepping its range
    as one batch with no exchange; one all-gather of the per-world centroids
    at the end.  Total work is fixed: strong scaling."""
    import torch
    from melon3d_b200 import shard
    W = args.batch_worlds
    counts = [harness.batch_world_bodies(k) for k in range(W)]
    ranges = shard.partition_worlds(counts, d.world)
    s0, s1 = ranges[d.rank]
    scenes, mine, batch = _batch_from(lib, range(s0, s1))
    for s in scenes:
        s.close()
    if batch:
        lib.m3d_world_step(batch, 1.0 / 60.0, args.substeps)
    torch.cuda.synchronize()
    d.barrier()
    dev = 0.0
    for _ in range(args.batch_steps):
        if batch:
            lib.m3d_world_step(batch, 1.0 / 60.0, args.substeps)
            dev += lib.m3d_gpu_last_step_device_ms(batch)
    torch.cuda.synchronize()
    d.barrier()
    cent = _world_centroids(lib, batch, s1 - s0) if batch else np.zeros((0, 3))
    full = shard.gather_world_results(cent, ranges, d.rank, d.pg, device="cuda")
    dev_max = d.reduce(dev, "MAX")
    if batch:
        lib.m3d_world_destroy(batch)
    work = int(sum(counts)) * args.substeps * args.batch_steps
    return {"workload": "%d batched worlds sharded by world over %d GPUs" % (W, d.world), "scaling": "strong",
            "ranges": ranges, "bodies": int(sum(counts)), "steps": args.batch_steps,
            "value": work / (dev_max / 1000.0), "unit": "body-substeps/s", "ms_per_step": dev_max / args.batch_steps,
            "gathered_worlds": int(full.shape[0]), "centroid_checksum": float(np.nansum(full))}


def measure_asleep(lib, args, ref_lib):
    """Fixed per-step cost of fully asleep scenes: 2,400 / 8,000 / 18,000
    unit boxes in 2-box stacks on a grid, stepped until every body sleeps and
    the sleeping-world fast path is on, then timed (host wall time per step
    through the C API, 200 steps); the reference steps the same scenes."""
    out = {"workload": "fully asleep 2-box stacks (2,400 / 8,000 / 18,000 unit boxes), 60 Hz x 4 substeps",
           "unit": "ms/step", "scenes": []}
    cores = os.cpu_count() or 1
    for dims in ((40, 30, 2), (80, 50, 2), (150, 60, 2)):
        row = {"boxes": dims[0] * dims[1] * dims[2]}
        for name, l, workers in (("gpu", lib, 0), ("reference", ref_lib, cores)):
            if l is None or (name == "reference" and args.no_cpu_baseline):
                continue
            sc = harness.Scene(l, harness.SETTLED_STACKS, 1, *dims, workers=workers)
            for _ in range(120):
                sc.run(1, args.substeps)
                if l.m3d_world_profile(sc.world).awakeBodyCount == 0 and (
                        name == "reference" or l.m3d_gpu_fast_path_steps(sc.world) > 0):
                    break
            _, wall_ms, _ = sc.run(200, args.substeps)
            row[name + "_ms_per_step"] = wall_ms / 200
            if name == "gpu":
                row["gpu_fast_path_steps"] = int(l.m3d_gpu_fast_path_steps(sc.world))
            sc.close()
        out["scenes"].append(row)
    out["reference_sample"] = "reference release build, workerCount=%d, 200 steps after the scene sleeps" % cores
    return out


def _incline_batch(lib, W):
    scenes = [harness.Scene(lib, harness.INCLINE, k) for k in range(W)]
    ids = [s.dynamic_ids() for s in scenes]
    arr = (C.c_void_p * W)(*[s.world for s in scenes])
    batch = lib.m3d_gpu_batch_create(arr, W)
    slots = [[lib.m3d_gpu_batch_first_body(batch, k) + i.index for i in ids[k]] for k in range(W)]
    for s in scenes:
        s.close()
    return batch, slots


def measure_adjoint(lib, args):
    """Differentiable batch: 1024 incline worlds x 64 bodies, 120 steps at
    60 Hz x 4 substeps; loss = sum over worlds of |centroid - target|^2 with
    seeded targets; gradients of v0, masses, friction, restitution from
    m3d_gpu_step_backward with checkpoints every 10 steps.  Forward alone
    against forward with the tape plus the backward, on the same worlds.
    Roofline of the backward: the tape's bytes (every record is read at
    least once) over the backward's device time."""
    W, steps = args.adjoint_worlds, args.adjoint_steps
    # untimed warm-up: the first batch of this shape pays the arena's allocations
    batch, slots = _incline_batch(lib, W)
    for _ in range(3):
        lib.m3d_world_step(batch, 1.0 / 60.0, args.substeps)
    lib.m3d_world_destroy(batch)
    batch, slots = _incline_batch(lib, W)
    bodies = sum(len(s) for s in slots)
    fwd_dev = fwd_wall = 0.0
    for _ in range(steps):
        t = time.perf_counter()
        lib.m3d_world_step(batch, 1.0 / 60.0, args.substeps)
        fwd_wall += (time.perf_counter() - t) * 1000.0
        fwd_dev += lib.m3d_gpu_last_step_device_ms(batch)
    lib.m3d_world_destroy(batch)
    batch, slots = _incline_batch(lib, W)
    assert lib.m3d_gpu_tape_begin(batch, 10) == 0
    rec_dev = rec_wall = 0.0
    for _ in range(steps):
        t = time.perf_counter()
        lib.m3d_world_step(batch, 1.0 / 60.0, args.substeps)
        rec_wall += (time.perf_counter() - t) * 1000.0
        rec_dev += lib.m3d_gpu_last_step_device_ms(batch)
    why = C.create_string_buffer(200)
    supported = lib.m3d_gpu_tape_supported(batch, why, 200) == 1
    tape_bytes = lib.m3d_gpu_tape_bytes(batch)
    n = lib.m3d_gpu_body_capacity(batch)
    pos = (C.c_float * (3 * n))()
    lib.m3d_gpu_read_poses(batch, pos, None, n)
    p = np.frombuffer(pos, dtype=np.float32).reshape(n, 3).astype(np.float64)
    targets = np.random.default_rng(5).normal(size=(W, 3))
    dpos = np.zeros((n, 3), np.float32)
    loss = 0.0
    for k, s in enumerate(slots):
        r = p[s].mean(axis=0) - targets[k]
        loss += float(r @ r)
        dpos[s] = (2.0 * r / len(s)).astype(np.float32)
    g = {k: np.zeros((n, 3) if k in ("pos", "vel", "ang") else ((n, 4) if k == "rot" else n), np.float32)
         for k in ("pos", "rot", "vel", "ang", "mass", "mu", "e")}
    fp = C.POINTER(C.c_float)
    lib.m3d_gpu_profiler_reset(b"*")
    t = time.perf_counter()
    rc = lib.m3d_gpu_step_backward(batch, dpos.ctypes.data_as(fp), None, None, None,
                                   *[g[k].ctypes.data_as(fp) for k in ("pos", "rot", "vel", "ang", "mass", "mu", "e")], n)
    bwd_wall = (time.perf_counter() - t) * 1000.0
    timed = _profiler_table(lib)
    lib.m3d_gpu_profiler_reset(b"")
    lib.m3d_world_destroy(batch)
    bwd_dev = sum(ms for _, ms in timed.values())
    top = sorted(timed.items(), key=lambda kv: -kv[1][1])[:5]
    peak, source = _peaks()
    achieved = tape_bytes / (bwd_dev / 1000.0) / 1e9 if bwd_dev > 0 else 0.0
    work = bodies * args.substeps * steps
    total = rec_wall + bwd_wall
    gv = np.concatenate([g["vel"][s] for s in slots]).astype(np.float64)
    finite = np.isfinite(gv)
    return {"workload": "%d incline worlds x 64 bodies (cubes and spheres 0.1-0.3 m, v0~N(0,1), mu~U[0.2,0.9], "
                        "e~U[0,0.3]), %d steps, checkpoints every 10" % (W, steps),
            "bodies": bodies, "steps": steps, "status": rc, "tape_supported": supported,
            "value": work / (total / 1000.0), "unit": "body-substeps/s",
            "forward_ms": fwd_wall, "forward_device_ms": fwd_dev,
            "recorded_forward_ms": rec_wall, "recorded_forward_device_ms": rec_dev, "backward_ms": bwd_wall,
            "backward_kernel_ms": bwd_dev,
            "backward_top_kernels": [{"kernel": k, "launches": v[0], "ms": v[1]} for k, v in top],
            "fwd_plus_adjoint_over_forward": total / fwd_wall,
            "roofline": {"bound": "hbm", "kernel": "backward (all kernels, event-timed)", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                         "bytes_per_launch": tape_bytes, "model": "tape bytes (records, tables, checkpoints) read "
                                                                 "at least once by the backward",
                         "peak_source": source + " (burst copy bandwidth)"},
            "loss": loss, "grad_v0_finite_fraction": float(finite.mean()),
            "grad_v0_norm": float(np.linalg.norm(gv[finite])), "grad_v0_median_abs": float(np.median(np.abs(gv)))}


def main():
    args = parse()
    d = Dist(args.gpus)
    if args.impl == "reference":
        if d.rank == 0:
            res, why = run_reference_sample(args.steps, args.warmup, args)
            if res is None:
                print(json.dumps({"impl": "reference", "unavailable": why}))
            else:
                line = {"metric": "body-substeps/s", "value": res["value"], "unit": "body-substeps/s",
                        "n_gpus": d.world, "steps": args.steps, "warmup": args.warmup,
                        "ms_per_step": res["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                        "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
                        "config": bench_config(args, d.world),
                        "cpu_baseline": {k: res[k] for k in ("value", "unit", "cores", "kind", "sample")},
                        "e2e": {"value": res["value"], "unit": "body-substeps/s", "h2d_bytes_per_step": 0,
                                "d2h_bytes_per_step": 0}}
                print(json.dumps(line))
        d.barrier()
        d.close()
        return

    import torch
    torch.cuda.set_device(d.local)
    lib = api.load_gpu()
    if args.only_adjoint:
        if d.rank == 0:
            print(json.dumps(measure_adjoint(lib, args)))
        d.barrier()
        d.close()
        return
    scene = harness.Scene(lib, harness.RAIN, 2, args.bodies, args.churn, 0)
    world = scene.world
    scene.run(args.preroll + max(args.warmup, 3), args.substeps)
    flush_buf = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB

    clocks = Clocks(d.local)
    d.barrier()
    torch.cuda.synchronize()
    tm = Timed(lib, world, args.roofline_kernels.split(","), args.substeps)
    clocks.start()
    body_substeps = 0
    for _ in range(args.steps):
        flush_l2(flush_buf)
        torch.cuda.synchronize()
        bs = [0]
        tm.step(lambda: bs.__setitem__(0, scene.run(1, args.substeps)[0]))
        body_substeps += bs[0]
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = lib.m3d_gpu_profiler_launches()
    h2d, d2h = C.c_longlong(0), C.c_longlong(0)
    lib.m3d_gpu_profiler_bytes(C.byref(h2d), C.byref(d2h))
    roofs = tm.rooflines()
    status = lib.m3d_gpu_status(world)
    d.barrier()
    dev_ms_max = d.reduce(tm.dev, "MAX")
    wall_ms_max = d.reduce(tm.wall, "MAX")
    total_bs = d.reduce(body_substeps, "SUM")

    cpu = None
    if d.rank == 0 and d.world == 1 and not args.no_cpu_baseline:
        cpu, _ = run_reference_sample(args.steps, args.warmup, args, seconds_cap=args.cpu_baseline_seconds)
        if cpu is not None:
            cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}

    variants = None
    if not args.no_variants:
        if d.world == 1:
            ref_lib = api.bind(C.CDLL(REF_RELEASE_LIB)) if os.path.exists(REF_RELEASE_LIB) else None
            variants = {"batched": measure_batch(lib, args, ref_lib), "pile": measure_pile(lib, args, ref_lib),
                        "fwd_adjoint": measure_adjoint(lib, args), "asleep": measure_asleep(lib, args, ref_lib)}
        else:
            variants = {"batched_sharded": measure_batch_sharded(lib, args, d)}
    if d.rank == 0:
        line = {"metric": "body-substeps/s", "value": total_bs / (dev_ms_max / 1000.0), "unit": "body-substeps/s",
                "n_gpus": d.world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": dev_ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": bench_config(args, d.world),
                "e2e": {"value": total_bs / (wall_ms_max / 1000.0), "unit": "body-substeps/s",
                        "h2d_bytes_per_step": h2d.value // max(args.steps, 1),
                        "d2h_bytes_per_step": d2h.value // max(args.steps, 1),
                        "ms_per_step": wall_ms_max / args.steps},
                "roofline": roofs[0] if roofs else None, "roofline_others": roofs[1:], "cpu_baseline": cpu,
                "gpu_launches": launches, "clocks": clk, "status": status, "variants": variants}
        print(json.dumps(line))
    scene.close()
    d.barrier()
    d.close()


if __name__ == "__main__":
    main()
