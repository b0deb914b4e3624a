#!/usr/bin/env python
"""Benchmark of the curvilinear velocity-stress RK4 step on B200.

One "step" is one accepted classic-RK4 time step of a whole shot (four fused stage kernels, the
device-side diagnostics/acceptance verdict and the receiver recording).  Default workload: the
5001x2001 2D elastic curvilinear shot (seeded terrain and layers, 30-cell CFS-PML, explosive
source), plain FP64.  Metric: grid-point RK4 updates per second (Mpt-updates/s), computational
nodes (absorber strips included, ghosts excluded) x steps / time.

    python bench.py [--gpus N --steps K --warmup W] [--impl swl|reference] [--workload NAME]

* value      : device time (CUDA events on the engine's stream) of K steps, state resident in HBM
* e2e        : the same K steps through the public session API (Simulation2D.advance): forcing
               uploads from pinned host memory and receiver traces downloaded every step, wall time
* roofline   : algorithmic HBM bytes of the stage kernels / their event-timed duration
* cpu_baseline: the reference's own CPU solver (oracle/_ref, built from its sources) on a bounded
               sample of the same shot, all host threads
* N > 1      : one independent shot per GPU (shots never exchange data); weak scaling
"""
from __future__ import annotations

import os

# More hardware work queues than the default 8, so that the serving leg's per-shot streams do not
# share queues and serialise behind one another; it must be set before the CUDA context exists.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

import argparse
import ctypes as C
import importlib.util
import json
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG_DIR = ROOT / "seiswavelab--curvilinear_b200"
METRIC = "Mpt-updates/s & shots/hr: batched FP32 vs plain FP64 on B200 at <=1e-4 trace L2"
UNIT = "Mpt-updates/s"


def load_package():
    if "swl_b200" in sys.modules:
        return sys.modules["swl_b200"]
    spec = importlib.util.spec_from_file_location("swl_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["swl_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def workload(name: str, precision: int) -> tuple[dict, str]:
    import importlib
    W = importlib.import_module("swl_b200.workloads")
    if name == "curvilinear_large":
        return W.curvilinear_large(precision=precision), "2D elastic curvilinear 5001x2001 h=2 m, seeded terrain (60 m relief), 5 layers, explosive source 10 m deep, 30-cell CFS-PML, 1000 receivers"
    if name == "small":
        return W.curvilinear_large(precision=precision, nx=2001, nz=801), "2D elastic curvilinear 2001x801 (profiling size of curvilinear_large)"
    if name == "plain_small":
        return W.plain_small(precision=precision), "2D elastic 500x200 flat, 3 layers, surface force, 20-cell CFS-PML"
    if name == "gsls_medium":
        return W.gsls_medium(precision=precision), "2D GSLS (3 mechanisms) 2001x801, 40 m sinusoidal terrain, 30-cell CFS-PML"
    if name == "elastic_3d":
        return W.elastic_3d(precision=precision), "3D nine-field elastic 400x288x200 h=10 m, DEM terrain, 3 layers, 20-cell sponge"
    if name == "elastic_3d_cpml":
        return (W.elastic_3d(precision=precision, absorber=1),
                "3D nine-field elastic 400x288x200 h=10 m, DEM terrain, 3 layers, 20-cell CFS-PML slabs")
    if name == "gsls_3d":
        return (W.elastic_3d(precision=precision, mechanisms=3),
                "3D GSLS (3 mechanisms, 27 fields) 400x288x200 h=10 m, DEM terrain, 3 layers, 20-cell sponge")
    if name == "small_3d":
        return (W.elastic_3d(precision=precision, nx=200, ny=144, nz=100),
                "3D nine-field elastic 200x144x100 (profiling size of elastic_3d)")
    raise SystemExit(f"unknown workload {name}")


def source_scale_2d(p: dict) -> float:
    # src/two_d/CurvilinearSolver2D.cpp:558-561: (moment or force per length) / h^2
    amp = p.get("momentPerLength", 2e6) if int(p.get("sourceKind", 0)) == 1 else p.get("forcePerLength", 2e5)
    return amp / (p["spacing"] ** 2)


def measured_hbm_peak() -> tuple[float, str]:
    path = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(path.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class UtilSampler:
    """nvidia-smi GPU utilization (percent of time a kernel was running) every 100 ms."""

    def __init__(self, gpu: int):
        self.gpu, self.values, self.proc, self.thread = gpu, [], None, None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", "--query-gpu=utilization.gpu",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return self

        def read():
            for line in self.proc.stdout:
                try:
                    self.values.append(float(line.strip()))
                except ValueError:
                    pass
        self.thread = threading.Thread(target=read, daemon=True)
        self.thread.start()
        return self

    def stop(self) -> float | None:
        if not self.proc:
            return None
        self.proc.terminate()
        self.proc.wait()
        return float(np.mean(self.values)) if self.values else None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while running."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu, self.lines, self.proc, self.thread = gpu, [], None, None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=lambda: [self.lines.append(l) for l in self.proc.stdout], daemon=True)
        self.thread.start()

    def wait_first(self, timeout: float = 5.0):
        t0 = time.time()
        while self.proc and not self.lines and time.time() - t0 < timeout:
            time.sleep(0.02)

    def stop(self) -> dict | None:
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "samples": len(sm), "reasons": sorted(reasons)}


def cpu_baseline(params: dict, dim: int, steps: int, warmup: int, keep: bool = False):
    """The reference's own CPU solver on a bounded sample of the same shot, all host threads.
    With `keep`, also returns the run's final fields and records (the reference's answer for
    the same warmup + steps, against which the GPU path's error is reported)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    threads = min(64, os.cpu_count() or 1)
    run = O.run_reference_2d if dim == 2 else O.run_reference_3d
    ref = O.REF2D if dim == 2 else O.REF3D
    if not ref.exists():
        return (None, None) if keep else None
    p = dict(params)
    p["maxSteps"] = warmup + steps
    p["precision"] = 0
    r = run(p, steps=steps, threads=threads, dump_mesh=False, warmup=warmup)
    pts = float(np.prod([int(r[k]) - 6 for k in (("nx", "nz") if dim == 2 else ("nx", "ny", "nz"))]))
    sec = float(r["runMs"]) / 1e3
    base = {"value": pts * steps / sec / 1e6, "unit": UNIT, "cores": int(r["threads"]), "kind": "reference",
            "ms_per_step": float(r["msPerStep"]),
            "sample": f"{steps} timed steps after {warmup} warm-up of the same shot (reference CPU solver, FP64, "
                      f"{int(r['threads'])} OpenMP threads); {float(r['msPerStep']):.1f} ms/step, init {float(r['initMs'])/1e3:.1f} s"}
    return (base, r) if keep else base


def error_vs_reference(S, params: dict, dim: int, ref: dict, device: int) -> dict:
    """Trace and wavefield error of the GPU path against the reference CPU solver's own run of the
    same shot and step count (the run the CPU baseline timed): FP64 plain and FP32 chosen form."""
    steps = int(ref["steps"])
    nfields = int(ref["fieldCount"]) if dim == 2 else 9
    comps = ("Vx", "Vz") if dim == 2 else ("Vx", "Vy", "Vz")
    R, Sm = int(ref["receivers"]), int(ref["samples"])
    want_tr = [ref[f"traces{c}"].reshape(R, Sm) for c in comps]
    want_f = [ref[f"field{f}"] for f in range(nfields)]

    def rel(a, b):
        den = float(np.linalg.norm(b))
        return float(np.linalg.norm(a - b) / den) if den > 0 else float(np.linalg.norm(a - b))

    out = {"steps": steps, "reference": "reference CPU solver (oracle/_ref), FP64, same shot and steps"}
    for prec, key in ((0, "fp64"), (1, "fp32")):
        sim = (S.Simulation2D if dim == 2 else S.Simulation3D)(dict(params, precision=prec), device=device)
        sim.advance(steps)
        got_tr = list(sim.records())
        got_f = [sim.field(f) for f in range(nfields)]
        tr = max(rel(a, b) for a, b in zip(got_tr, want_tr))
        fl = max(rel(a, b) for a, b in zip(got_f, want_f) if np.any(b))
        res = {"trace_rel_l2": tr, "field_rel_l2": fl}
        if prec == 0:
            res["bitwise"] = bool(all(np.array_equal(a, b) for a, b in zip(got_tr, want_tr)) and
                                  all(np.array_equal(a, b) for a, b in zip(got_f, want_f)))
        out[key] = res
        sim.close()
    return out


def traffic_from_profiles(workload_name: str, dtype: str):
    path = ROOT / "profiles" / "traffic.json"
    try:
        t = json.loads(path.read_text())
        return t.get(f"{workload_name}:{dtype}")
    except Exception:
        return None


def reference_gpu(params: dict, steps: int, warmup: int) -> dict | None:
    """The reference's own CUDA engine (src/two_d/CudaEngine2D.cu, built from its sources for
    sm_100a) on the same 2D shot, FP64 and FP32: production advance() with its per-step stats and
    receiver readback, timed by the reference driver after a warm-up."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    if not O.REF2D_CUDA.exists():
        return None
    out = {"engine": "reference CudaEngine (src/two_d/CudaEngine2D.cu), sm_100a build", "steps": steps, "warmup": warmup}
    for prec, key in ((0, "fp64"), (1, "fp32")):
        p = dict(params)
        p["maxSteps"] = warmup + steps
        p["precision"] = prec
        r = O.run_reference_2d(p, steps=steps, threads=1, dump_mesh=False, warmup=warmup, backend="cuda", timeout=600)
        pts = float((int(r["nx"]) - 6) * (int(r["nz"]) - 6))
        sec = float(r["runMs"]) / 1e3
        out[key] = {"value": pts * steps / sec / 1e6, "unit": UNIT, "ms_per_step": float(r["msPerStep"])}
    return out


def max_over_ranks(x: float, dist, device: str) -> float:
    """The largest value of x over all ranks: a multi-GPU job takes as long as its slowest rank."""
    if not dist:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(points: int, steps: int, ms: float, world: int) -> float:
    """Whole-job Mpt-updates/s: each of `world` ranks advances its own shot of `points` nodes by
    `steps` steps, and the job takes `ms` (the slowest rank's time)."""
    return world * points * steps / (ms * 1e-3) / 1e6


def time_engine(swl, sim, dim, params, steps, warmup, torch, dist, rank):
    """Device time of `steps` engine steps on torch's current stream; returns (ms, profile)."""
    L = swl.library()
    eng = C.c_void_p(sim.engine_handle())
    info = sim.info()
    dt, f = info["dt"], float(params["frequency"])
    stream = torch.cuda.Stream()  # a real stream: handle 0 would mean "the engine's own stream"
    acc = C.c_int32()
    set_stream = L.swl2d_set_stream if dim == 2 else L.swl3d_set_stream
    swl._check(set_stream(eng, C.c_void_p(stream.cuda_stream)))
    # trace and forcing tables sized for the timed batch: it allocates nothing and records no graph
    swl._check((L.swl2d_reserve if dim == 2 else L.swl3d_reserve)(eng, max(steps, warmup)))

    def run(first, n):
        if dim == 2:
            st = L.swl2d_advance(eng, first, n, dt, f, source_scale_2d(params), 3.0 / f, C.byref(acc))
        else:
            st = L.swl3d_advance(eng, first, n, dt, f, 3.0 / f, C.byref(acc))
        swl._check(st)

    step = info["step"]
    run(step, warmup)  # a multiple of 8: the timed batch replays the CUDA graph the warm-up recorded
    step += warmup
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    run(step, steps)
    end.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = start.elapsed_time(end)
    step += steps
    prof = swl.Profile()
    if dim == 2:
        swl._check(L.swl2d_profile(eng, step, 8, dt, f, source_scale_2d(params), C.byref(prof)))
    else:
        swl._check(L.swl3d_profile(eng, step, 8, dt, f, C.byref(prof)))
    swl._check(set_stream(eng, None))
    out = prof.as_dict()
    if dim == 2:
        out["layout"] = swl.layout2d(eng)  # strip width, rows per block, the tuned segment, interior CTAs
    return ms, out


def serving_leg(args, device: int) -> dict:
    """Shots/hour and latency of a seeded request stream: batched FP32 through the request loop
    (requests submitted at their Poisson arrival times, concurrent shots on one GPU) versus the
    plain FP64 path running the same requests one after another."""
    import importlib
    W = importlib.import_module("swl_b200.workloads")
    S = importlib.import_module("swl_b200.session")
    V = importlib.import_module("swl_b200.server")
    # The full mix arrives at 20 requests/s.  Shrinking every shot by scale^2 (grid) x steps (time)
    # shrinks the offered work per second by the same factor, so the arrival rate is raised by it:
    # the scaled stream then loads the GPU as the full stream does (throughput-bound), rather than
    # leaving it idle between arrivals.
    rate = args.serving_rate or 20.0 / (args.serving_scale ** 2 * args.serving_steps)
    reqs = W.serving_mix(n=args.serving_requests, rate=rate, seed=5, scale=args.serving_scale,
                         steps_scale=args.serving_steps)
    a0 = reqs[0]["arrival"]

    def kind(r):
        return "3d" if r["dim"] == 3 else "2d_gsls" if r["params"].get("attenuation") else "2d_elastic"

    # Untimed warm-up: one 16-step shot of each kind in each precision, so that neither leg loads
    # kernel modules inside its timed region (CUDA loads them lazily, on first use); a serving
    # process pays that once, not per stream.
    warmed = set()
    for r in reqs:
        if kind(r) in warmed:
            continue
        warmed.add(kind(r))
        for prec in (0, 1):
            p = dict(r["params"], precision=prec, maxSteps=16)
            if r["dim"] == 2:
                p["segmentRule"] = prec  # the batched (FP32) form picks segments by rule
            w = (S.Simulation2D if r["dim"] == 2 else S.Simulation3D)(p, device=device)
            w.advance(16)
            w.close()
    # batched FP32
    srv = V.Server(device=device, batch_steps=args.serving_batch, max_active=args.serving_active,
                   build_threads=max(2, min(8, (os.cpu_count() or 4) // 2)), scheduler_threads=args.serving_schedulers,
                   persistent=args.serving_persistent, persistent_ctas=args.serving_persistent_ctas)
    util = UtilSampler(device).start()
    t0 = time.perf_counter()
    ids = []
    for r in reqs:
        delay = (r["arrival"] - a0) - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        ids.append(srv.submit(dict(r["params"], precision=1), r["dim"]))
    srv.drain()
    util32 = util.stop()
    st = [srv.status(i) for i in ids]
    failed = [s["error"] for s in st if s["state"] != "done"]
    lat32 = np.array([s["finish_s"] - s["submit_s"] for s in st])
    build32 = np.array([s["run_s"] - s["start_s"] for s in st])  # host model build + engine creation
    gpu32 = np.array([s["finish_s"] - s["run_s"] for s in st])   # first batch to last batch
    span32 = max(s["finish_s"] for s in st) - min(s["submit_s"] for s in st)
    rec32 = [srv.records(i) for i in ids]
    stats = srv.stats()
    srv.close()
    # sequential (same requests, arrival order, one at a time): plain FP64 and, to separate the
    # precision's share of the gain from the batching's, FP32
    def sequential(precision):
        service, records, init = [], [], []
        by_kind = {}
        u = UtilSampler(device).start()
        for r in reqs:
            t = time.perf_counter()
            sim = (S.Simulation2D if r["dim"] == 2 else S.Simulation3D)(dict(r["params"], precision=precision), device=device)
            init.append(time.perf_counter() - t)
            info = sim.info()
            sim.advance(info["total_steps"])
            records.append(sim.records())
            del sim
            service.append(time.perf_counter() - t)
            k = by_kind.setdefault(kind(r), {"shots": 0, "init_s": 0.0, "run_s": 0.0, "node_steps": 0.0})
            nodes = (info["nx"] - 6) * (info["nz"] - 6) * ((info["ny"] - 6) if r["dim"] == 3 else 1)
            k["shots"] += 1
            k["init_s"] += init[-1]
            k["run_s"] += service[-1] - init[-1]
            k["node_steps"] += nodes * info["total_steps"]
        for k in by_kind.values():
            k["mpt_per_s"] = k["node_steps"] / k["run_s"] / 1e6 if k["run_s"] > 0 else None
        return service, records, float(np.sum(init)), u.stop(), by_kind
    batched = {"shots_per_hour": len(reqs) / span32 * 3600, "p50_s": float(np.percentile(lat32, 50)),
               "p99_s": float(np.percentile(lat32, 99)), "makespan_s": span32, "peak_running": stats["peak_running"],
               "failed": failed, "mean_build_s": float(build32.mean()), "mean_run_s": float(gpu32.mean()),
               "gpu_util_pct": util32, "scheduler_threads": args.serving_schedulers, "max_active": args.serving_active,
               "persistent_2d": args.serving_persistent, "persistent_ctas_per_sm": args.serving_persistent_ctas}
    if args.serving_batched_only:
        return {"requests": len(reqs), "batched_fp32": batched}
    service, rec64, init64, util64, kinds64 = sequential(0)
    if args.serving_fp32_sequential:
        service32, _, init32, util32s, kinds32 = sequential(1)
    else:
        service32, init32, util32s, kinds32 = [], None, None, None
    finish, lat64, clock = [], [], 0.0
    for r, s in zip(reqs, service):
        start = max(clock, r["arrival"] - a0)
        clock = start + s
        lat64.append(clock - (r["arrival"] - a0))
    span64 = clock
    errs = []
    for a, b in zip(rec32, rec64):
        num = sum(float(np.sum((x - y) ** 2)) for x, y in zip(a, b))
        den = sum(float(np.sum(y ** 2)) for y in b)
        errs.append((num / den) ** 0.5 if den > 0 else 0.0)
    shots = len(reqs)
    return {
        "requests": shots, "mix": f"seeded (seed 5) Poisson {rate:g}/s (the full mix's 20/s times the work shrink "
                                  f"factor); 80% 2D elastic/GSLS, 20% 3D; grid edges x{args.serving_scale}, "
                                  f"steps x{args.serving_steps} of the full mix",
        "batched_fp32": batched,
        "sequential_fp64": {"shots_per_hour": shots / span64 * 3600, "p50_s": float(np.percentile(lat64, 50)),
                            "p99_s": float(np.percentile(lat64, 99)), "makespan_s": span64,
                            "sum_init_s": init64, "gpu_util_pct": util64, "by_kind": kinds64,
                            "latency_model": "the requests ran one after another; each one's measured service time is "
                                             "queued at its arrival time (FIFO, one GPU) to give its latency"},
        "sequential_fp32": {"sum_service_s": float(np.sum(service32)), "sum_init_s": init32, "gpu_util_pct": util32s,
                            "by_kind": kinds32} if args.serving_fp32_sequential else None,
        "shots_per_hour_ratio": (shots / span32) / (shots / span64),
        "max_trace_rel_l2_fp32_vs_fp64": max(errs), "median_trace_rel_l2_fp32_vs_fp64": float(np.median(errs)),
    }


def persistent_leg(args, device: int) -> dict:
    """Throughput of the persistent multi-shot launch (swl2d_queue_launch) against the same shots'
    own batches running concurrently on their own streams: FP32 2D shots of the serving mix, 64
    steps per round, unforced (scale 0; the arithmetic and traffic do not depend on the values)."""
    import ctypes as C
    import importlib
    swl = load_package()
    W = importlib.import_module("swl_b200.workloads")
    S = importlib.import_module("swl_b200.session")
    reqs = [r for r in W.serving_mix(n=4 * args.persistent_shots, rate=100.0, seed=5, scale=args.serving_scale,
                                     steps_scale=args.serving_steps) if r["dim"] == 2]
    out = {"steps_per_round": 64, "rounds": 3, "unit": "Mpt-updates/s"}
    for label, gsls in (("elastic", False), ("gsls3", True)):
        group = [r for r in reqs if bool(r["params"].get("attenuation")) == gsls][:args.persistent_shots]
        sims = [S.Simulation2D(dict(r["params"], precision=1, segmentRule=1), device=device) for r in group]
        engs = []
        for sm in sims:
            e = swl.Engine2D.__new__(swl.Engine2D)
            e._h = C.c_void_p(sm.engine_handle())
            engs.append(e)
        info = [sm.info() for sm in sims]
        nodes = sum((i["nx"] - 6) * (i["nz"] - 6) for i in info)
        dts, freqs = [i["dt"] for i in info], [r["params"]["frequency"] for r in group]
        q = swl.Queue2D(1, device)

        def streams(first):
            for e, d, f in zip(engs, dts, freqs):
                e.launch(first, 64, d, f, 0.0)
            for e in engs:
                e.wait()

        def queued(first):
            q.launch(engs, first, 64, dts, freqs, 0.0)
            q.wait()
            for e in engs:
                e.wait()

        res = {"shots": len(engs), "nodes": nodes}
        for name, fn in (("own_streams", streams), ("persistent", queued)):
            fn(0)  # warm-up (module load, tables)
            t = time.perf_counter()
            for k in range(3):
                fn(64 * (k + 1))
            res[name] = nodes * 64 * 3 / (time.perf_counter() - t) / 1e6
        res["ratio"] = res["persistent"] / res["own_streams"]
        out[label] = res
        q.close()
        for e in engs:
            e._h = C.c_void_p()  # the sessions own the engines
        del sims
    return out


def gpu_arm(args):
    import torch
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as D
        torch.cuda.set_device(local)
        D.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = D
    torch.cuda.set_device(local)
    swl = load_package()
    import importlib
    S = importlib.import_module("swl_b200.session")
    dim = 3 if args.workload in ("elastic_3d", "elastic_3d_cpml", "gsls_3d", "small_3d") else 2
    Sim = S.Simulation2D if dim == 2 else S.Simulation3D
    peak, peak_src = measured_hbm_peak()

    def measure(precision):
        params, desc = workload(args.workload, precision)
        t0 = time.perf_counter()
        sim = Sim(params, device=local)
        init_s = time.perf_counter() - t0
        info = sim.info()
        pts = (info["nx"] - 6) * (info["nz"] - 6) if dim == 2 else (info["nx"] - 6) * (info["ny"] - 6) * (info["nz"] - 6)
        sampler = ClockSampler(local) if precision == 0 and rank == 0 else None
        if sampler:
            sampler.start()
            sampler.wait_first()  # the sampler is up before the timed region starts
        ms, prof = time_engine(swl, sim, dim, params, args.steps, args.warmup, torch, dist, rank)
        clocks = sampler.stop() if sampler else None
        ms = max_over_ranks(ms, dist, "cuda")
        stage_ms = sum(prof["stage_ms"])
        achieved = prof["bytes_per_step"] / (stage_ms * 1e-3) / 1e9
        res = {"value": job_throughput(pts, args.steps, ms, world), "ms_per_step": ms / args.steps, "points": pts,
               "init_s": init_s, "profile": prof, "desc": desc, "params": params, "clocks": clocks,
               "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                            "traffic": traffic_from_profiles(args.workload, "f64" if precision == 0 else "f32"),
                            "kernel": "fused RK stage kernels (4 per step)", "peak_source": peak_src,
                            "bytes_per_step": prof["bytes_per_step"], "stage_ms_per_step": stage_ms,
                            "bytes_rule": "17F + 4M per node-step plus 17 words per CFS-PML memory (algorithmic)",
                            "kahan_bytes_per_step": prof["extra_bytes_per_step"],
                            "frac_with_kahan": (prof["bytes_per_step"] + prof["extra_bytes_per_step"]) / (stage_ms * 1e-3) / 1e9 / peak}}
        return sim, res

    sim64, r64 = measure(0)
    # e2e: the same K steps through the public session API (host forcing upload and trace
    # download inside the timed region), from a reset shot.
    sim64.reset()
    sim64.advance(args.warmup)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    sim64.advance(args.steps)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, dist, "cuda")
    info = sim64.info()
    nrec = info["receivers"]
    e2e = {"value": world * r64["points"] * args.steps / e2e_s / 1e6, "unit": UNIT,
           "h2d_bytes_per_step": 3 * 8, "d2h_bytes_per_step": (2 if dim == 2 else 3) * 8 * nrec,
           "api": "Simulation.advance (session C ABI), wall time"}
    del sim64
    r32 = None
    if not args.no_fp32:
        sim32, r32 = measure(1)
        del sim32
    base = parity = parity_long = None
    if rank == 0 and world == 1 and not args.no_cpu:
        base, ref_run = cpu_baseline(r64["params"], dim, args.cpu_steps, 1, keep=True)
        if ref_run is not None:
            parity = error_vs_reference(S, r64["params"], dim, ref_run, local)
            del ref_run
        if args.parity_steps > 0:
            # a run long enough for the waves to cross the grid (the headline shot's 7 steps reach only the
            # source's neighbourhood): the 500x200 plain workload, the reference CPU solver on all threads
            sys.path.insert(0, str(ROOT / "oracle"))
            import oracle as O
            import importlib
            W = importlib.import_module("swl_b200.workloads")
            pp = W.plain_small(precision=0, steps=args.parity_steps)
            ref_long = O.run_reference_2d(pp, steps=args.parity_steps, threads=min(64, os.cpu_count() or 1), dump_mesh=False)
            parity_long = error_vs_reference(S, pp, 2, ref_long, local)
            parity_long["workload"] = "plain_small (500x200 h=2, 20-cell CFS-PML, surface force)"
            del ref_long
    ref_gpu = None
    if rank == 0 and world == 1 and dim == 2 and not args.no_ref_gpu:
        ref_gpu = reference_gpu(r64["params"], args.ref_gpu_steps, 2)
    serving = None
    if rank == 0 and world == 1 and args.serving_requests > 0:
        serving = serving_leg(args, local)
    persistent = None
    if rank == 0 and world == 1 and args.persistent_shots > 0:
        persistent = persistent_leg(args, local)

    if rank == 0:
        line = {
            "metric": METRIC, "value": r64["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r64["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded terrain/layers/sources, PCG64)",
            "config": {"workload": args.workload, "description": r64["desc"], "points": r64["points"],
                       "precision": "fp64 plain", "l2": "inputs larger than L2 (resident state and model > 2 GB)",
                       "parallelism": "one independent shot per GPU" if world > 1 else "single shot",
                       "init_s": round(r64["init_s"], 3)},
            "roofline": r64["roofline"], "e2e": e2e, "gpu_launches": int(args.steps * r64["profile"]["launches_per_step"]),
            "clocks": r64["clocks"], "cpu_baseline": base, "error_vs_reference": parity,
            "error_vs_reference_long": parity_long,
        }
        if r32:
            line["fp32"] = {"value": r32["value"], "unit": UNIT, "ms_per_step": r32["ms_per_step"],
                            "roofline": r32["roofline"], "speedup_vs_fp64": r32["value"] / r64["value"],
                            "profile": r32["profile"]}
        if ref_gpu:
            line["reference_gpu"] = ref_gpu
        if serving:
            line["serving"] = serving
        if persistent:
            line["persistent_launch"] = persistent
        line["profile_fp64"] = r64["profile"]
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def reference_arm(args):
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return
    load_package()
    dim = 3 if args.workload in ("elastic_3d", "elastic_3d_cpml", "gsls_3d", "small_3d") else 2
    params, desc = workload(args.workload, 0)
    steps = min(args.steps, args.cpu_steps)
    warm = min(args.warmup, 3)  # untimed steps before the sample (a CPU step of the 5001x2001 shot is ~0.9 s)
    base = cpu_baseline(params, dim, steps, warm)
    if base is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU solver binaries (oracle/_ref) are not built"}))
        return
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": base["value"], "unit": UNIT, "n_gpus": 0, "steps": steps,
        "warmup": warm, "ms_per_step": base["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded terrain/layers/sources, PCG64)",
        "config": {"workload": args.workload, "description": desc, "precision": "fp64 plain"},
        "cpu_baseline": base, "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=8)
    ap.add_argument("--impl", choices=["swl", "reference"], default="swl")
    ap.add_argument("--workload", default="curvilinear_large",
                    choices=["curvilinear_large", "small", "plain_small", "gsls_medium", "elastic_3d", "elastic_3d_cpml",
                             "gsls_3d", "small_3d"])
    ap.add_argument("--cpu-steps", type=int, default=6, help="timed steps of the reference CPU sample")
    ap.add_argument("--parity-steps", type=int, default=600,
                    help="steps of the long parity run against the reference (500x200 plain workload; 0: skip)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true", help="skip timing the reference's own CUDA engine")
    ap.add_argument("--ref-gpu-steps", type=int, default=10, help="timed steps of the reference CUDA engine")
    ap.add_argument("--no-fp32", action="store_true")
    ap.add_argument("--serving-requests", type=int, default=48, help="requests of the serving leg (0: skip)")
    ap.add_argument("--persistent-shots", type=int, default=24,
                    help="FP32 2D shots per group in the persistent-launch vs own-stream comparison (0: skip)")
    ap.add_argument("--serving-persistent", type=int, default=0,
                    help="1: the 2D shots of the batched form advance together in one persistent launch per round; "
                         "2: the elastic 2D shots only; 0: every shot on its own stream")
    ap.add_argument("--serving-persistent-ctas", type=int, default=-1,
                    help="resident CTAs per SM of a persistent launch (0 all, n>0 at most n, n<0 all but -n)")
    ap.add_argument("--serving-scale", type=float, default=0.5, help="grid-edge scale of the serving mix")
    ap.add_argument("--serving-steps", type=float, default=0.25, help="step-count scale of the serving mix")
    ap.add_argument("--serving-batch", type=int, default=64, help="steps per batch of a served shot")
    ap.add_argument("--serving-schedulers", type=int, default=2, help="server threads driving the running shots")
    ap.add_argument("--serving-fp32-sequential", type=int, default=1,
                    help="also run the requests one after another in FP32 (separates precision from batching; 0: skip)")
    ap.add_argument("--serving-batched-only", action="store_true",
                    help="run only the batched leg (to compare serving settings; no ratio)")
    ap.add_argument("--serving-active", type=int, default=32, help="shots built or running at once (0: memory-bound only)")
    ap.add_argument("--serving-rate", type=float, default=0.0,
                    help="arrivals per second (0: 20/s of the full mix scaled by the work shrink factor)")
    args = ap.parse_args()
    if args.warmup < 3:
        raise SystemExit("--warmup must be >= 3")
    # Batches run as CUDA graphs of 8 steps keyed by the step phase; a warm-up that is a multiple
    # of 8 leaves the timed batch on the graph the warm-up already recorded (no capture inside the
    # timed region).  The line reports the warm-up actually run.
    args.warmup = (args.warmup + 7) // 8 * 8
    if args.impl == "reference":
        reference_arm(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
