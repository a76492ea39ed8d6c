#!/usr/bin/env python
"""Benchmark of the Yee/CPML/ADE/TF-SF hot path on B200.

Default workload: the large dispersive configuration -- 512^3 cells on a
graded 1-3 mm mesh plus 12 CPML layers per face (536^3 swept cells), 30 % of
the volume in 2-pair pole-residue blocks, a soft Ez dipole at the centre --
built from seeded synthetic inputs.  A step is one whole leapfrog step (E
half: curl + CPML + ADE + sources; H half: curl + CPML + sources; probe
gather).  Metric: Gcell-updates/s = swept cells x steps / s.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank runs an independent replica on its own GPU
(the hot path is single-rank; "replicas only"), time is the max over ranks and
value is the sum of the replicas' cell updates over that time.

--impl reference times the reference algorithm's CPU implementation (the
C++ restatement in oracle/, OpenMP over all host cores) on the same workload
(its set-up untimed, a bounded number of whole steps timed); the Fortran
reference itself cannot be built here.
"""
from __future__ import annotations

import argparse
import ctypes as C
import gc
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

METRIC = "Gcell-upd/s"
CONFIGS = {
    # name: (generator, kwargs, workload label)
    "dispersive_large": ("dispersive_large", {}, "512^3 graded 1-3 mm, CPML 12 (536^3 swept), 30% 2-pair pole-residue, soft Ez dipole"),
    "plain_mid": ("plain_mid", {}, "256^3 dx 5 mm, CPML 12, lossy sphere + 20 PEC/dielectric blocks, TF/SF plane wave"),
    "plain_small": ("plain_small", {}, "64^3 dx 1 cm, CPML 10, TF/SF plane wave"),
    "batched": (None, {}, "64 instances (seed 6): edges log-U[32,160] per axis, CPML 8, 1-6 dielectric blocks, "
                          "seeded plane wave, steps U{500..3000}"),
    "served": (None, {}, "Poisson stream (seed 7): edges log-U[48,256], CPML 10, 0-2 pole-residue blocks, soft dipole, "
                         "4-32 probes, steps U{500..4000} x steps_scale"),
}
CPU_STEPS = 3  # whole steps of the CPU baseline on the benchmarked case (about 0.5 s each on 16 cores)
NOMINAL_HBM_GBS = 8000.0  # the nominal B200 HBM3e figure the fractions are also reported against


def env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def make_case(config: str, n: int | None, steps_needed: int):
    from semba_fdtd_b200 import casegen, read_case
    gen, kw, label = CONFIGS[config]
    kw = dict(kw)
    if n is not None:
        kw["n"] = n
        if config == "dispersive_large":
            kw["edge"] = (max(4, n // 16), max(8, n // 4))
    d = Path(tempfile.mkdtemp(prefix="semba_bench_"))
    path = getattr(casegen, gen)(d, **kw)
    pb = read_case(path)
    pb.nsteps = max(pb.nsteps, steps_needed)
    if n is not None:
        label = f"{label}; scaled to {n} cells per axis"
    return pb, label


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.out = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "50"], stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        # nvidia-smi takes a moment to start: wait for its first sample so the
        # (short) timed region that follows is sampled
        t0 = time.perf_counter()
        while self.proc and time.perf_counter() - t0 < 5.0:
            try:
                if Path(self.out.name).read_text().strip():
                    break
            except Exception:
                pass
            time.sleep(0.02)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        try:
            rows = [r.split(",") for r in Path(self.out.name).read_text().splitlines() if r.strip()]
        except Exception:
            rows = []
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in rows for q in range(4) if len(r) > 5 + q and r[5 + q].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_hbm_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(kernel: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary."""
    p = ROOT / "profiles" / "ncu_traffic.json"
    try:
        t = json.loads(p.read_text())
        return t.get(kernel)
    except Exception:
        return None


def cpu_model() -> str:
    try:
        for ln in Path("/proc/cpuinfo").read_text().splitlines():
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def cpu_oracle(pb, steps: int, warmup: int = 0, budget_s: float = 120.0, single_thread_step: bool = True,
               keep_fields: bool = False):
    """The oracle (the reference algorithm restated in C++, OpenMP over all
    host cores) on the benchmarked case itself: set-up untimed, `warmup`
    untimed steps, then up to `steps` whole steps timed (fewer if they exceed
    budget_s), then one more step on a single thread.  Returns a dict with
    the rates, the sample description and (keep_fields) the six fields after
    the timed steps."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    threads = os.cpu_count() or 1
    o = oracle.Oracle(pb, threads=threads)
    try:
        if warmup:
            o.step(warmup)
        t0 = time.perf_counter()
        done = 0
        while done < steps:
            o.step(1)
            done += 1
            if time.perf_counter() - t0 > budget_s:
                break
        t_all = time.perf_counter() - t0
        fields = [o.field(c) for c in range(6)] if keep_fields else None
        rate1 = None
        if single_thread_step:
            o.set_threads(1)
            t1 = time.perf_counter()
            o.step(1)
            rate1 = pb.swept_cells / (time.perf_counter() - t1) / 1e9
    finally:
        o.close()
    return {"rate": pb.swept_cells * done / t_all / 1e9, "threads": threads, "steps": done, "warmup": warmup,
            "rate_1thread": rate1, "cpu_model": cpu_model(), "fields": fields,
            "sample": f"the benchmarked case itself ({pb.swept_cells} swept cells), {done} whole steps after "
                      f"{warmup} untimed, set-up untimed, FP32 oracle (-O2, no FMA contraction), OpenMP"}


def run_reference(args):
    rank, _, world = env_rank()
    if rank != 0:
        return
    pb, label = make_case(args.config, args.n, args.steps + args.warmup + 8)
    r = cpu_oracle(pb, max(1, args.steps), warmup=min(max(0, args.warmup), 2), budget_s=150.0)
    rate = r["rate"]
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": "Gcell-upd/s", "n_gpus": args.gpus,
            "steps": r["steps"], "warmup": r["warmup"], "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {"workload": label, "swept_cells": pb.swept_cells},
            "cpu_baseline": {"value": rate, "unit": "Gcell-upd/s", "cores": r["threads"], "kind": "port",
                             "sample": r["sample"], "cpu_model": r["cpu_model"], "value_1thread": r["rate_1thread"]},
            "e2e": {"value": rate, "unit": "Gcell-upd/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    rank, local, world = env_rank()
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from semba_fdtd_b200 import Solver, _lib
    lib = _lib.load("exact")
    if lib.sgpu_select_device(local) != 0:
        raise SystemExit("cannot select CUDA device")
    K, W = args.steps, max(3, args.warmup)
    pb, label = make_case(args.config, args.n, K + W + 8)
    cells = pb.swept_cells

    def barrier():
        if dist:
            dist.barrier()

    def allmax(x):
        if not dist:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def allsum(x):
        if not dist:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())

    bufs = None if args.quick else e2e_buffers(pb, lib)
    # ---- device-resident throughput ------------------------------------
    s = Solver(pb, probe_capacity=max(1024, K + W + CPU_STEPS + 8), kernel_family=args.family)
    # the first CPU_STEPS steps are kept for the parity check against the
    # oracle's run of the same steps (rank 0, not timed)
    check_fields = None
    if not args.quick and not args.skip_cpu and rank == 0:
        s.step(CPU_STEPS)
        check_fields = [s.field(c) for c in range(6)]
    s.step(W)
    s.synchronize()
    ms = C.c_float()
    barrier()
    with ClockSampler(local) as clk:
        rc = lib.sgpu_elapsed_steps(s.handle, s.n, K, C.byref(ms))
    if rc:
        raise SystemExit(f"sgpu_elapsed_steps failed: {lib.sgpu_last_error(s.handle).decode()}")
    s.n += K
    t_ms = allmax(ms.value)
    barrier()
    per_step = C.c_int()
    lib.sgpu_kernels_per_step(s.handle, C.byref(per_step))
    launches = per_step.value * K + (K + 31) // 32 + 1
    # ---- per-phase device times and algorithmic bytes (roofline) -------
    phases = (C.c_float * 6)()
    s._drain()
    rc = lib.sgpu_profile_steps(s.handle, s.n, K, phases)
    if rc:
        raise SystemExit(f"sgpu_profile_steps failed: {lib.sgpu_last_error(s.handle).decode()}")
    s.n += K
    moved6 = (C.c_double * 6)()
    lib.sgpu_algorithmic_bytes(s.handle, moved6)
    bytes6 = (C.c_double * 6)()
    lib.sgpu_compulsory_bytes(s.handle, bytes6)
    names = ["efield_curl_cpml", "edispersive_ade", "sources_e", "hfield_curl_cpml", "sources_h", "probes"]
    fe, fh = ("k_tma_efield", "k_tma_hfield") if args.family == 1 else ("k_efield", "k_hfield")
    kern = [fe, "k_ade", "k_sources", fh, "k_sources", "k_probes"]
    avg_ms = [phases[q] / K for q in range(6)]
    dom = int(np.argmax(avg_ms))
    peak, peak_kind = measured_hbm_peak()
    achieved = bytes6[dom] / (avg_ms[dom] * 1e-3) / 1e9 if avg_ms[dom] > 0 else None
    achieved_moved = moved6[dom] / (avg_ms[dom] * 1e-3) / 1e9 if avg_ms[dom] > 0 else None
    finite = s.check_finite()
    s.close()

    # ---- end to end through the C ABI with host buffers -----------------
    e2e = None if args.quick else run_e2e(pb, K, lib, args.family, bufs)

    value = allsum(cells * K) / (t_ms * 1e-3) / 1e9
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    step_bytes = sum(bytes6[q] for q in range(6))
    step_moved = sum(moved6[q] for q in range(6))
    step_s = t_ms / K * 1e-3
    line = {"metric": METRIC, "value": value, "unit": "Gcell-upd/s", "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": t_ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": label, "swept_cells": cells, "parallelism": f"replicas{world}",
                       "l2": ("inputs larger than L2 (fields alone %.1f GB)" % (cells * 24 / 1e9)
                              if cells * 24 > 126e6 else
                              "inputs fit in L2 (fields %.0f MB); no flush between steps" % (cells * 24 / 1e6)),
                       "build": "-fmad=false (bit-exact)",
                       "field_kernels": "TMA-pipelined" if args.family == 1 else "register-marching"},
            "step_roofline": {"bytes": step_bytes, "achieved": step_bytes / step_s / 1e9,
                              "frac": step_bytes / step_s / 1e9 / peak,
                              "frac_nominal": step_bytes / step_s / 1e9 / NOMINAL_HBM_GBS, "moved_bytes": step_moved,
                              "frac_moved": step_moved / step_s / 1e9 / peak,
                              "bytes_definition": "compulsory (sgpu_compulsory_bytes): 60 B per cell + 8 B per psi "
                                                  "point + (8 + 32 x stored poles) B per pole-residue node; moved "
                                                  "(sgpu_algorithmic_bytes): what the kernels' design reads and writes"},
            "roofline": {"bound": "hbm", "kernel": kern[dom], "phase": names[dom], "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
                         "frac_nominal": (achieved / NOMINAL_HBM_GBS) if achieved else None,
                         "traffic": ncu_traffic(kern[dom]), "algorithmic_bytes": bytes6[dom],
                         "achieved_moved": achieved_moved, "frac_moved": (achieved_moved / peak) if achieved_moved else None,
                         "moved_bytes": moved6[dom], "avg_ms": avg_ms[dom],
                         "phases_ms": dict(zip(names, avg_ms)), "phases_bytes": dict(zip(names, list(bytes6))),
                         "phases_moved_bytes": dict(zip(names, list(moved6)))},
            "clocks": clk.summary(), "gpu_launches": launches, "finite": finite, "e2e": e2e}
    try:
        if args.quick or args.skip_cpu:
            raise RuntimeError("skipped (--quick / --skip-cpu)")
        r = cpu_oracle(pb, CPU_STEPS, budget_s=60.0, keep_fields=check_fields is not None)
        line["cpu_baseline"] = {"value": r["rate"], "unit": "Gcell-upd/s", "cores": r["threads"], "kind": "port",
                                "sample": r["sample"], "cpu_model": r["cpu_model"], "value_1thread": r["rate_1thread"]}
        if check_fields is not None and r["fields"] is not None and r["steps"] == CPU_STEPS:
            same = all(a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))
                       for a, b in zip(check_fields, r["fields"]))
            line["parity"] = {"steps": CPU_STEPS, "fields_bit_equal_to_oracle": bool(same),
                              "what": "all six fields after the first steps of this run, bit patterns, against the "
                                      "oracle's run of the same steps (tests/test_parity_full.py covers more steps)"}
    except Exception as ex:  # the baseline is reported, not the target
        line["cpu_baseline"] = {"value": None, "unit": "Gcell-upd/s", "cores": os.cpu_count(), "kind": "port",
                                "sample": f"failed: {ex}"}
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def e2e_buffers(pb, lib):
    """The caller's host buffers of the end-to-end leg: the initial fields
    (zeros, a fresh start) and the final fields, in pinned memory.  They are
    made before any timing (7.4 GB at 536^3 take a few seconds to pin), so
    the end-to-end leg does not start on a GPU that idled meanwhile."""
    from semba_fdtd_b200 import _lib
    desc, keep = pb.to_desc()
    plan = C.c_void_p()
    if lib.sgpu_host_plan(C.byref(desc), 1, C.byref(plan)):
        raise SystemExit("sgpu_host_plan failed")
    a6, s6, q6 = (_lib.Lim * 6)(), (_lib.Lim * 6)(), (_lib.Lim * 6)()
    lib.sgpu_host_info(plan, C.byref(C.c_double()), C.byref(C.c_int()), a6, s6, q6)
    lib.sgpu_destroy(plan)
    shapes = [(a.ze - a.zi + 1, a.ye - a.yi + 1, a.xe - a.xi + 1) for a in a6]
    init = [_lib.pinned_empty(sh, np.float32) for sh in shapes]
    final = [_lib.pinned_empty(sh, np.float32) for sh in shapes]
    for a in init + final:
        a.fill(0.0)
    return init, final


def run_e2e(pb, K, lib, family, bufs):
    """Host problem -> device (set-up, media from the problem description,
    initial fields from pinned host buffers) -> K steps -> probe traces and
    final fields back into pinned host buffers."""
    from semba_fdtd_b200 import Solver
    init, final = bufs
    t0 = time.perf_counter()
    s = Solver(pb, probe_capacity=max(1024, K + 8), kernel_family=family)
    t_setup = time.perf_counter()
    h2d = 0  # sgpu_host_create builds the media matrices on the device from the region list
    for c in range(6):
        s.upload_field(c, init[c])
        h2d += init[c].nbytes
    t_h2d = time.perf_counter()
    s.step(K)
    s.synchronize()
    t_steps = time.perf_counter()
    tr = s.probes()
    d2h = tr.nbytes
    for c in range(6):
        s.field(c, out=final[c])
        d2h += final[c].nbytes
    t_end = time.perf_counter()
    t = t_end - t0
    s.close()
    return {"value": pb.swept_cells * K / t / 1e9, "unit": "Gcell-upd/s", "h2d_bytes_per_step": h2d / K,
            "d2h_bytes_per_step": d2h / K, "seconds": t,
            "breakdown_s": {"setup": t_setup - t0, "field_upload": t_h2d - t_setup,
                            "steps": t_steps - t_h2d, "download": t_end - t_steps},
            "includes": "host set-up and device-built media matrices, initial-field upload from pinned host "
                        "memory, K graph steps, probe and final-field download into pinned host memory"}


def _stream_batched(n_inst: int, seed: int = 6):
    from semba_fdtd_b200 import casegen, read_case
    rng = np.random.default_rng(seed)
    d = Path(tempfile.mkdtemp(prefix="semba_batched_"))
    return [read_case(casegen.batch_instance(d, q, rng)) for q in range(n_inst)]


def _stream_served(n_req: int, rate: float, steps_scale: float, seed: int = 7):
    from semba_fdtd_b200 import casegen, read_case
    from semba_fdtd_b200.serve import Request, poisson_arrivals
    rng = np.random.default_rng(seed)
    d = Path(tempfile.mkdtemp(prefix="semba_served_"))
    arr = poisson_arrivals(n_req, rate, seed)
    reqs = []
    for q in range(n_req):
        steps = max(1, int(round(int(rng.integers(500, 4001)) * steps_scale)))
        pb = read_case(casegen.served_request(d, q, rng, steps=steps))
        reqs.append(Request(rid=q, arrival=float(arr[q]), problem=pb, nsteps=steps))
    return reqs


def _cells_steps(pb, nsteps):
    return pb.swept_cells * (nsteps + 1)


def run_batched(args):
    """The 64-instance stream as one batch (autotuned, 32-step graph chunks)
    against the same instances one at a time through Solver.  Both arms
    include host set-up, device upload and probe read-back; solves/s is
    instances / wall time."""
    from concurrent.futures import ThreadPoolExecutor

    from semba_fdtd_b200 import Solver
    from semba_fdtd_b200.batch import Batch, Plan
    rank, local, world = env_rank()
    if rank != 0:
        return
    pbs = _stream_batched(args.instances)
    work = sum(_cells_steps(pb, pb.nsteps) for pb in pbs)
    # Python's cyclic garbage collector stays off while either arm is timed,
    # so a collection pass over the stream's objects lands in neither
    gc.collect()
    gc.disable()
    # plain arm: one solve at a time
    t0 = time.perf_counter()
    for pb in ([] if args.skip_plain else pbs):
        with Solver(pb, probe_capacity=pb.nsteps + 1) as s:
            s.step(pb.nsteps + 1)
            s.probes()
    t_plain = time.perf_counter() - t0 if not args.skip_plain else float("nan")
    # batched arm
    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        marks = {}
        with ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 1)) as pool:  # host set-up in parallel
            plans = list(pool.map(Plan, pbs))
        marks["plan"] = time.perf_counter() - t0
        arena = int(sum(p.footprint for p in plans) * 1.05) + (64 << 20)
        with Batch(arena, len(pbs) + 1, kernel_family=args.batch_family) as b:
            # most steps first (or in stream order, or most work first), a
            # first group, then 32-step chunks queued between the remaining
            # set-ups (an instance is set up on its own stream while the
            # queued steps of the others run), then the tuner with every
            # instance live, so its trial steps run at full occupancy
            if args.batch_order == "longest":
                plans = sorted(plans, key=lambda p: -(p.nsteps + 1) * p.problem.swept_cells)
            elif args.batch_order == "steps":
                # most steps first: the solves that set the length of the run
                # start first (a stable sort, stream order among equals)
                plans = sorted(plans, key=lambda p: -p.nsteps)
            first = 8
            slots = [b.add(p) for p in plans[:first]]
            for q, p in enumerate(plans[first:]):
                if q % args.batch_advance_every == 0:
                    b.advance(32)
                slots.append(b.add(p))
            marks["add"] = time.perf_counter() - t0
            chunks, ctas = b.autotune(2)
            marks["tune"] = time.perf_counter() - t0
            live = sum(1 for x in slots if not b.done(x))
            phases = b.profile(8)  # real steps, per-phase device time of the live instances
            dev_ms = 0.0
            while any(not b.done(x) for x in slots):
                left = max(b.info(x)[1] - b.info(x)[0] for x in slots)
                dev_ms += b.elapsed(min(256, max(32, left)))
            marks["steps"] = time.perf_counter() - t0
            for x in slots:
                b.probes(x)
            marks["read"] = time.perf_counter() - t0
        t_batch = time.perf_counter() - t0
        marks["closed"] = t_batch
    gc.enable()
    line = {"metric": "solves/s", "value": len(pbs) / t_batch, "unit": "solves/s", "n_gpus": 1, "steps": None,
            "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "impl": "batched",
            "config": {"workload": CONFIGS["batched"][2], "instances": len(pbs), "cell_updates": work,
                       "arena_bytes": arena, "tuned_chunks": chunks, "tuned_ctas_per_sm": ctas,
                       "batched_arm_marks_s": marks,
                       "field_kernels": "TMA-pipelined persistent" if args.batch_family == 1 else "register-marching"},
            "plain_one_at_a_time": {"solves_per_s": len(pbs) / t_plain if not args.skip_plain else None,
                                    "seconds": None if args.skip_plain else t_plain,
                                    "gcell_upd_s": None if args.skip_plain else work / t_plain / 1e9},
            "batched": {"seconds": t_batch, "gcell_upd_s": work / t_batch / 1e9, "device_step_ms_total": dev_ms,
                        "device_gcell_upd_s": work / (dev_ms * 1e-3) / 1e9 if dev_ms else None,
                        "phase_ms_8_steps": dict(zip(["e_field", "ade", "e_sources", "h_field", "h_sources",
                                                      "probes"], phases)), "phase_live_instances": live},
            "speedup_vs_plain": None if args.skip_plain else t_plain / t_batch, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def run_served(args):
    """A Poisson stream (step counts scaled) served with continuous batching
    against the same stream served one solve at a time through Solver."""
    from semba_fdtd_b200.serve import Server, run_plain
    rank, local, world = env_rank()
    if rank != 0:
        return
    reqs = _stream_served(args.requests, args.rate, args.steps_scale)
    work = sum(_cells_steps(r.problem, r.nsteps) for r in reqs)
    plain = run_plain(reqs, keep_traces=False).summary()
    for r in reqs:
        r.plan = None
    with ClockSampler(local) as clk:
        srv = Server(arena_bytes=int(args.arena_gb * (1 << 30)), max_instances=512, chunk=32, backfill=32,
                     autotune=True)
        try:
            st = srv.run(reqs, keep_traces=False).summary()
        finally:
            srv.close()
    line = {"metric": "solves/s", "value": st["solves_per_s"], "unit": "solves/s", "n_gpus": 1, "steps": None,
            "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "impl": "served",
            "config": {"workload": CONFIGS["served"][2], "requests": len(reqs), "rate_per_s": args.rate,
                       "steps_scale": args.steps_scale, "cell_updates": work, "hbm_budget_gb": args.arena_gb},
            "served": st, "plain_one_at_a_time": plain,
            "speedup_vs_plain": (st["solves_per_s"] / plain["solves_per_s"]) if plain["solves_per_s"] else None,
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="dispersive_large", choices=list(CONFIGS))
    ap.add_argument("--n", type=int, default=None, help="scale the configuration (cells per axis)")
    ap.add_argument("--family", type=int, default=1, choices=[0, 1],
                    help="field kernels: 1 TMA-pipelined (default), 0 register-marching")
    ap.add_argument("--quick", action="store_true", help="skip the end-to-end and CPU-baseline legs (profiling runs)")
    ap.add_argument("--skip-cpu", action="store_true", help="skip the CPU-baseline leg and its parity check")
    ap.add_argument("--instances", type=int, default=64, help="batched: instances in the stream")
    ap.add_argument("--skip-plain", action="store_true", help="batched: leave out the one-at-a-time arm (profiling)")
    ap.add_argument("--batch-order", default="steps", choices=["longest", "steps", "stream"],
                    help="batched: order in which the instances join the batch")
    ap.add_argument("--batch-advance-every", type=int, default=4,
                    help="batched: a 32-step chunk is queued after this many instance set-ups")
    ap.add_argument("--batch-family", type=int, default=1, choices=[0, 1],
                    help="batched: field kernels, 1 TMA-pipelined persistent (default), 0 register-marching")
    ap.add_argument("--requests", type=int, default=160, help="served: requests in the stream")
    ap.add_argument("--rate", type=float, default=32.0, help="served: Poisson arrival rate (1/s)")
    ap.add_argument("--steps-scale", type=float, default=0.25, help="served: scale of the drawn step counts")
    ap.add_argument("--arena-gb", type=float, default=150.0, help="served: HBM budget of the arena")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.config == "batched":
        run_batched(args)
    elif args.config == "served":
        run_served(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
