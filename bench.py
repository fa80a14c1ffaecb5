#!/usr/bin/env python
"""Body-substeps/s of the GPU world on the streaming mixed-rain workload.

Workload (one "step"): the 20,000-body streaming mixed rain (spheres,
capsules and boxes in thirds over a 100x60x100 m volume, seeded synthetic
data) advanced by one m3d_world_step at 60 Hz with 4 substeps, after the 200
lowest dynamic bodies are destroyed and 200 new ones spawned through the C
API.  Metric: body-substeps/s = dynamic bodies x substeps per step, summed
over the timed steps, divided by the time.

  value  device time of the steps: CUDA events on the world's stream around
         each m3d_world_step (uploads of the step's new bodies included);
  e2e    host wall time of the same steps through the C ABI, churn included:
         the H2D copies of the spawned bodies, the D2H pose read used to pick
         the lowest bodies and the per-step event/counter reads.
The L2 (126 MB) is flushed between timed steps by a 256 MiB write.

--impl reference times the reference's own CPU implementation (the
reference library built from its sources with its release flags) on the
same workload with all host threads.  N > 1 (torchrun) runs one independent
replica per GPU (a single world does not shard); value is the sum of the
replicas' work over the slowest replica's time.
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


# Algorithmic bytes per step of the kernels reported against the roofline:
# each field a kernel must read or write, counted once (fp32 SoA).
ROOFLINE_MODELS = {
    # serial islands: the whole substep loop of every serial island
    "kSolveSerial": ("HBM bytes per serial-island body, contact and point per substep", _serial_bytes),
    # free-body islands: every substep integrates and reconstructs each body
    "kSolveFree": ("HBM bytes per free body per substep", lambda c, sub: c["freeIslands"] * 300.0 * sub),
    # narrowphase: per live contact the two body indices, flags, two poses,
    # two cached poses, point count (~150 B); regenerated pairs also write
    # their manifold (~4 x 132 B) - counted as the cached case (a floor)
    "kNarrowphase": ("HBM bytes per contact", lambda c, sub: c["contactCount"] * 150.0),
}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=120)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["gpu", "reference"], default="gpu")
    p.add_argument("--bodies", type=int, default=20000)
    p.add_argument("--churn", type=int, default=200)
    p.add_argument("--substeps", type=int, default=4)
    p.add_argument("--roofline-kernels", default="kSolveSerial,kSolveFree,kNarrowphase")
    p.add_argument("--cpu-baseline-seconds", type=float, default=15.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-variants", action="store_true",
                   help="skip the batched-worlds and large-pile measurements")
    p.add_argument("--batch-worlds", type=int, default=4096)
    p.add_argument("--batch-steps", type=int, default=40)
    p.add_argument("--pile-steps", type=int, default=12)
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
    """The reference's CPU step on the same workload, all host threads."""
    if not os.path.exists(REF_RELEASE_LIB):
        return None, "oracle/_ref/libmelon3d_ref_fast.so not built"
    lib = api.bind(C.CDLL(REF_RELEASE_LIB))
    cores = os.cpu_count() or 1
    sc = harness.Scene(lib, harness.RAIN, 2, args.bodies, args.churn, 0, workers=cores)
    sc.run(warmup, args.substeps)
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
            "sample": "%d steps (after %d warm-up) of the same workload, reference release build, "
                      "workerCount=%d" % (done, warmup, cores), "ms_per_step": wall_total / max(done, 1)}, None


def _device_steps(lib, world, steps, substeps, bodies):
    """Steps through the C API: device time (CUDA events on the world's
    stream) and host wall time, in ms."""
    dev = 0.0
    t = time.perf_counter()
    for _ in range(steps):
        lib.m3d_world_step(world, 1.0 / 60.0, substeps)
        dev += lib.m3d_gpu_last_step_device_ms(world)
    wall = (time.perf_counter() - t) * 1000.0
    return dev, wall


def measure_pile(lib, args, ref_lib):
    """250,000-box settled pile (50x100x50 lattice), one giant island: the
    whole-GPU coloured solve.  Step 0 (3.1M contacts created) is untimed."""
    sc = harness.Scene(lib, harness.PILE, 3, 50, 100, 50)
    n = sc.sl.scn_dynamic_count(sc.handle)
    lib.m3d_world_step(sc.world, 1.0 / 60.0, args.substeps)
    lib.m3d_world_step(sc.world, 1.0 / 60.0, args.substeps)
    dev, wall = _device_steps(lib, sc.world, args.pile_steps, args.substeps, n)
    pr = lib.m3d_world_profile(sc.world)
    out = {"workload": "settled pile, 250,000 boxes (50x100x50 lattice, 1.02 m spacing, jitter), one giant island",
           "bodies": n, "steps": args.pile_steps, "value": n * args.substeps * args.pile_steps / (dev / 1000.0),
           "unit": "body-substeps/s", "ms_per_step": dev / args.pile_steps,
           "e2e": {"value": n * args.substeps * args.pile_steps / (wall / 1000.0), "ms_per_step": wall / args.pile_steps},
           "contacts": pr.contactCount, "touching": pr.touchingContactCount, "status": lib.m3d_gpu_status(sc.world)}
    sc.close()
    if ref_lib is not None and not args.no_cpu_baseline:
        cores = os.cpu_count() or 1
        rs = harness.Scene(ref_lib, harness.PILE, 3, 50, 100, 50, workers=cores)
        rs.run(1, args.substeps)  # contact creation
        bs, wall_ms, _ = rs.run(2, args.substeps)
        rs.close()
        out["cpu_baseline"] = {"value": bs / (wall_ms / 1000.0), "unit": "body-substeps/s", "cores": cores,
                               "kind": "reference", "sample": "2 steps after the first, reference release build, "
                                                               "workerCount=%d" % cores}
    return out


def measure_batch(lib, args, ref_lib):
    """4096 independent worlds (own ground, 16-512 bodies, 0-4 joints) in one
    batch, against the same worlds stepped one at a time."""
    W = args.batch_worlds
    scenes = [harness.Scene(lib, harness.BATCH_WORLD, k) for k in range(W)]
    bodies = sum(s.sl.scn_dynamic_count(s.handle) for s in scenes)
    arr = (C.c_void_p * W)(*[s.world for s in scenes])
    batch = lib.m3d_gpu_batch_create(arr, W)
    # one at a time: the first worlds stepped through the plain path
    solo_n, solo_steps = min(64, W), 10
    t = time.perf_counter()
    solo_bs = 0
    for s in scenes[:solo_n]:
        bs, _, _ = s.run(solo_steps, args.substeps)
        solo_bs += bs
    solo_rate = solo_bs / (time.perf_counter() - t)
    for s in scenes:
        s.close()
    lib.m3d_world_step(batch, 1.0 / 60.0, args.substeps)
    launches0 = lib.m3d_gpu_profiler_launches()
    dev, wall = _device_steps(lib, batch, args.batch_steps, args.substeps, bodies)
    launches = lib.m3d_gpu_profiler_launches() - launches0
    pos = (C.c_float * (3 * lib.m3d_gpu_body_capacity(batch)))()
    lib.m3d_gpu_read_poses(batch, pos, None, lib.m3d_gpu_body_capacity(batch))
    value = bodies * args.substeps * args.batch_steps / (dev / 1000.0)
    e2e = bodies * args.substeps * args.batch_steps / (wall / 1000.0)
    out = {"workload": "%d worlds, log-uniform 16-512 bodies each (rain shapes, own ground box, 0-4 ball/hinge "
                       "joints)" % W, "bodies": bodies, "steps": args.batch_steps, "value": value,
           "unit": "body-substeps/s", "ms_per_step": dev / args.batch_steps,
           "e2e": {"value": e2e, "ms_per_step": wall / args.batch_steps},
           "one_at_a_time": {"value": solo_rate, "unit": "body-substeps/s",
                             "sample": "%d worlds x %d steps through the plain GPU path" % (solo_n, solo_steps)},
           "speedup_vs_one_at_a_time": e2e / solo_rate, "gpu_launches_per_step": launches / args.batch_steps,
           "status": lib.m3d_gpu_status(batch)}
    lib.m3d_world_destroy(batch)
    if ref_lib is not None and not args.no_cpu_baseline:
        cores = os.cpu_count() or 1
        rn, rsteps = min(256, W), 5
        t = time.perf_counter()
        rbs = 0
        for k in range(rn):
            rs = harness.Scene(ref_lib, harness.BATCH_WORLD, k, workers=cores)
            bs, _, _ = rs.run(rsteps, args.substeps)
            rbs += bs
            rs.close()
        out["cpu_baseline"] = {"value": rbs / (time.perf_counter() - t), "unit": "body-substeps/s", "cores": cores,
                               "kind": "reference", "sample": "%d worlds x %d steps one after another (world "
                                                              "creation included), workerCount=%d" % (rn, rsteps, cores)}
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
    against forward with the tape plus the backward, on the same worlds."""
    W, steps = args.adjoint_worlds, args.adjoint_steps
    batch, slots = _incline_batch(lib, W)
    bodies = sum(len(s) for s in slots)
    fwd_dev, fwd_wall = _device_steps(lib, batch, steps, args.substeps, bodies)
    lib.m3d_world_destroy(batch)
    batch, slots = _incline_batch(lib, W)
    assert lib.m3d_gpu_tape_begin(batch, 10) == 0
    rec_dev, rec_wall = _device_steps(lib, batch, steps, args.substeps, bodies)
    why = C.create_string_buffer(200)
    supported = lib.m3d_gpu_tape_supported(batch, why, 200) == 1
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
    t = time.perf_counter()
    rc = lib.m3d_gpu_step_backward(batch, dpos.ctypes.data_as(fp), None, None, None,
                                   *[g[k].ctypes.data_as(fp) for k in ("pos", "rot", "vel", "ang", "mass", "mu", "e")], n)
    bwd_wall = (time.perf_counter() - t) * 1000.0
    lib.m3d_world_destroy(batch)
    work = bodies * args.substeps * steps
    total = rec_wall + bwd_wall
    gv = np.concatenate([g["vel"][s] for s in slots])
    return {"workload": "%d incline worlds x 64 bodies (cubes and spheres 0.1-0.3 m, v0~N(0,1), mu~U[0.2,0.9], "
                        "e~U[0,0.3]), %d steps, checkpoints every 10" % (W, steps),
            "bodies": bodies, "steps": steps, "status": rc, "tape_supported": supported,
            "value": work / (total / 1000.0), "unit": "body-substeps/s",
            "forward_ms": fwd_wall, "forward_device_ms": fwd_dev,
            "recorded_forward_ms": rec_wall, "recorded_forward_device_ms": rec_dev, "backward_ms": bwd_wall,
            "fwd_plus_adjoint_over_forward": total / fwd_wall,
            "loss": loss, "grad_v0_norm": float(np.linalg.norm(gv)),
            "grad_v0_median_abs": float(np.median(np.abs(gv)))}


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
                        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                        "ms_per_step": res["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                        "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
                        "config": {"workload": WORKLOAD, "variant": "plain", "parallelism": "replicas"},
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
    scene.run(max(args.warmup, 3), args.substeps)
    flush_buf = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB
    counters = (C.c_uint32 * 64)()

    clocks = Clocks(d.local)
    d.barrier()
    torch.cuda.synchronize()
    names = [k for k in args.roofline_kernels.split(",") if k in ROOFLINE_MODELS]
    lib.m3d_gpu_profiler_reset(",".join(names).encode())
    clocks.start()
    dev_ms = wall_ms = 0.0
    body_substeps = 0
    alg_bytes = {k: 0.0 for k in names}
    for _ in range(args.steps):
        flush_l2(flush_buf)
        torch.cuda.synchronize()
        bs, wall, _ = scene.run(1, args.substeps)
        dev_ms += lib.m3d_gpu_last_step_device_ms(world)
        wall_ms += wall
        body_substeps += bs
        n = lib.m3d_gpu_step_counters(world, counters, 64)
        c = {name: counters[i] for i, name in enumerate(COUNTER_NAMES[:n])}
        for k in names:
            alg_bytes[k] += ROOFLINE_MODELS[k][1](c, args.substeps)
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = lib.m3d_gpu_profiler_launches()
    h2d, d2h = C.c_longlong(0), C.c_longlong(0)
    lib.m3d_gpu_profiler_bytes(C.byref(h2d), C.byref(d2h))
    table = C.create_string_buffer(1 << 14)
    lib.m3d_gpu_profiler_table(table, 1 << 14)
    timed = {}
    for row in table.value.decode().splitlines():
        kname, kl, kms = row.split()
        timed[kname] = (int(kl), float(kms))
    status = lib.m3d_gpu_status(world)
    d.barrier()
    dev_ms_max = d.reduce(dev_ms, "MAX")
    wall_ms_max = d.reduce(wall_ms, "MAX")
    total_bs = d.reduce(body_substeps, "SUM")

    cpu = None
    if d.rank == 0 and d.world == 1 and not args.no_cpu_baseline:
        cpu, _ = run_reference_sample(args.steps, args.warmup, args, seconds_cap=args.cpu_baseline_seconds)
        if cpu is not None:
            cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}

    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    traffic = read_traffic()
    roofs = []
    for k in names:
        if k not in timed or timed[k][0] == 0:
            continue
        kl, kms = timed[k]
        avg_s = kms / 1000.0 / kl
        per_launch = alg_bytes[k] / kl
        achieved = per_launch / avg_s / 1e9
        roofs.append({"bound": "hbm", "kernel": k, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                      "frac": achieved / hbm_peak, "traffic": traffic.get(k),
                      "bytes_per_launch": per_launch, "avg_launch_us": avg_s * 1e6, "launches": kl,
                      "share_of_step": kms / max(dev_ms, 1e-9), "model": ROOFLINE_MODELS[k][0],
                      "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"})
    roofs.sort(key=lambda r: -r["share_of_step"])
    roof = roofs[0] if roofs else None
    variants = None
    if d.rank == 0 and d.world == 1 and not args.no_variants:
        ref_lib = api.bind(C.CDLL(REF_RELEASE_LIB)) if os.path.exists(REF_RELEASE_LIB) else None
        variants = {"batched": measure_batch(lib, args, ref_lib), "pile": measure_pile(lib, args, ref_lib),
                    "fwd_adjoint": measure_adjoint(lib, args)}
    if d.rank == 0:
        line = {"metric": "body-substeps/s", "value": total_bs / (dev_ms_max / 1000.0), "unit": "body-substeps/s",
                "n_gpus": d.world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": dev_ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": WORKLOAD, "variant": "plain", "bodies": args.bodies,
                           "churn_per_step": args.churn, "substeps": args.substeps, "hz": 60,
                           "l2": "flushed between timed steps (256 MiB write)",
                           "parallelism": "replicas" if d.world > 1 else "single world"},
                "e2e": {"value": total_bs / (wall_ms_max / 1000.0), "unit": "body-substeps/s",
                        "h2d_bytes_per_step": h2d.value // max(args.steps, 1),
                        "d2h_bytes_per_step": d2h.value // max(args.steps, 1),
                        "ms_per_step": wall_ms_max / args.steps},
                "roofline": roof, "roofline_others": roofs[1:], "cpu_baseline": cpu, "gpu_launches": launches,
                "clocks": clk,
                "status": status, "variants": variants}
        print(json.dumps(line))
    scene.close()
    d.barrier()
    d.close()


if __name__ == "__main__":
    main()
