#!/usr/bin/env python
"""Benchmark of the coupled D3Q19 NS + D3Q7 AD + LDF time step.

Workload (default): the 512x256x256 random sphere pack, FP32 populations,
BGK with obstacle bounce-back, NEQ velocity inlet u = 0.02, pressure outlet,
AD Dirichlet C = 1 / Neumann outlet, Langmuir LDF (q_max 5, K_L 1.5, k 0.05),
tau 0.6 / 0.55.  One bench "step" is one coupled time step over the whole
lattice; the metric is MLUPS = cells x steps / time / 1e6 (whole job: summed
over ranks, each rank advancing its own replica -- the step is not sharded).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Prints one JSON line on rank 0.  Timing: W untimed steps, then K steps between
CUDA events on the lattice's stream, bracketed by a barrier and
torch.cuda.synchronize(); max over ranks.  Every step reads and writes ~7 GB
of populations, far more than the 126 MB L2, so no flush is needed.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_CELL = {"f32": 216, "f16": 120, "bf16": 120, "f16q": 120, "f64": 432}   # algorithmic bytes per coupled cell update
BYTES_PER_POP = {"f32": 4, "f16": 2, "bf16": 2, "f16q": 2, "f64": 8}
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="sphere_pack", choices=["sphere_pack", "channel_small", "batch", "adjoint"])
    ap.add_argument("--samples", type=int, default=64, help="batch workload: number of samples")
    ap.add_argument("--precision", default="f32", choices=["f32", "f16", "bf16", "f16q", "f64"])
    ap.add_argument("--size", default=None, help="override lattice size, e.g. 256x128x128")
    ap.add_argument("--prefetch", type=int, default=None,
                    help="L2 prefetch distance of the step kernel in 256-cell blocks (0 off; default: the "
                         "library's choice, half a resident wave for f32 and none for the other forms)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--shard", action="store_true",
                    help="N > 1: cut the lattice into z-slabs, one per GPU, with a halo exchange, or (batch "
                         "workload) split the samples across the GPUs (strong scaling); default: N independent "
                         "replicas")
    ap.add_argument("--no-reference-cuda", action="store_true",
                    help="skip timing the reference's own CUDA build on the same workload")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip timing the other forms (FP16, BF16, FP16 + fixed-point AD, FP64) beside FP32")
    ap.add_argument("--pair-kernel", default="off", choices=["off", "direct", "staged"],
                    help="16-bit --precision: run the main workload on the opt-in pair layout with this kernel")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip timing the batching form (64 uneven samples) beside FP32")
    return ap.parse_args()


def make_problem(args):
    from fluidmaxxer_b200 import problems
    kw = {}
    if args.size:
        nx, ny, nz = (int(v) for v in args.size.lower().split("x"))
        kw = dict(nx=nx, ny=ny, nz=nz)
    return problems.sphere_pack(**kw) if args.workload == "sphere_pack" else problems.channel_small(**kw)


def workload_desc(p):
    d = {"workload": f"{p.name}", "cells": p.n_cells, "collision": p.collision, "isotherm": p.isotherm,
         "tau_ns": p.tau, "tau_ad": p.tau_ad if not hasattr(p.tau_ad, "shape") else "field",
         "inlet_u": p.u_in[0], "l2": "each step streams ~7 GB (> 126 MB L2); no flush needed"}
    if p.notes.get("slab_porosity") is not None:
        d["porosity"] = round(p.notes["slab_porosity"], 4)
        d["spheres"] = p.notes.get("spheres")
    return d


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def traffic_per_cell(precision):
    """DRAM bytes per cell of the fused kernel, from the committed ncu summary
    (dram__bytes_read.sum + dram__bytes_write.sum of one captured launch on a
    smaller case of the same workload, divided by its cell count)."""
    import glob
    import re
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "k_coupled_step_*.md"))):
        with open(path) as fh:
            m = re.search(rf"^dram_bytes_per_cell_{precision}:\s*([0-9.]+)", fh.read(), re.M)
        if m:
            return float(m.group(1))
    return None


class Clocks:
    """SM clock and throttle reasons sampled during the timed region: NVML queries
    (read only) from a background thread every 2 ms, one sample taken at start and
    one at stop, so even a region of a few milliseconds has samples; nvidia-smi
    polling when NVML is unavailable."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.tmp = None
        self.nvml = None
        self.samples = []
        self.thread = None
        self.running = False

    def _sample(self):
        import pynvml as N
        h = self.nvml
        self.samples.append((N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM),
                             N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM),
                             N.nvmlDeviceGetCurrentClocksEventReasons(h)))

    def _loop(self):
        while self.running:
            try:
                self._sample()
            except Exception:
                return
            time.sleep(0.002)

    def start(self):
        try:
            import threading

            import pynvml as N
            N.nvmlInit()
            idx = str(self.idx).strip()
            self.nvml = (N.nvmlDeviceGetHandleByIndex(int(idx)) if idx.isdigit()
                         else N.nvmlDeviceGetHandleByUUID(idx))
            self._sample()
            self.running = True
            self.thread = threading.Thread(target=self._loop, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.tmp, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.nvml is not None:
            self.running = False
            self.thread.join(timeout=5)
            try:
                self._sample()
            except Exception:
                pass
            sm = [float(c) for c, _, _ in self.samples]
            reasons = sorted({n for _, _, r in self.samples for n, bit in self.REASONS if r & bit})
            return {"sm_mhz": statistics.median(sm) if sm else None,
                    "sm_max_mhz": max(float(m) for _, m, _ in self.samples) if self.samples else None,
                    "reasons": reasons, "samples": len(self.samples), "source": "nvml"}
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.tmp.flush()
        rows = []
        with open(self.tmp.name) as fh:
            for line in fh:
                parts = [s.strip() for s in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.tmp.name)
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "source": "nvidia-smi"}


def time_reference_cpu(p, steps, warmup, budget_s):
    """The reference's own kernels (FP32 build, OpenMP over all host threads;
    the restated oracle where they were not built) on the workload: the
    largest z-slab of whole x-y planes (the whole lattice when it fits) whose
    warmup + steps take about budget_s.  Shared by the cpu_baseline leg of the
    B200 line and the reference arm, so both measure the same way."""
    import numpy as np

    from fluidmaxxer_b200.problems import Problem
    from oracle.oracle import Oracle, reference_available, reference_threads
    kind = "reference" if reference_available("f32") else "port"
    impl = "reference" if kind == "reference" else "restated"

    def slab(nz):
        q = Problem(**{k: getattr(p, k) for k in p.__dataclass_fields__})
        q.nz = nz
        q.solid = p.solid.reshape(p.nz, p.ny, p.nx)[:nz].reshape(-1).copy()
        q.region = None
        q.tau_ad = p.tau_ad if np.isscalar(p.tau_ad) else np.asarray(p.tau_ad).reshape(p.nz, -1)[:nz].reshape(-1)
        q.sample_every = 0
        return q

    nz0 = min(p.nz, 4)
    o = Oracle(slab(nz0), impl, "f32")
    t = time.perf_counter(); o.step(1); per_plane = (time.perf_counter() - t) / nz0
    o.close()
    nz = int(max(1, min(p.nz, budget_s / max(1, warmup + steps) / per_plane)))
    o = Oracle(slab(nz), impl, "f32")
    o.step(warmup)
    t = time.perf_counter(); o.step(steps); el = time.perf_counter() - t
    o.close()
    cells = p.nx * p.ny * nz
    cores = reference_threads() if kind == "reference" else os.cpu_count()
    what = "the whole lattice" if nz == p.nz else f"a {p.nx}x{p.ny}x{nz} z-slab"
    sample = (f"{what} of {p.name}, {warmup} + {steps} coupled steps, FP32 build of the reference kernels, "
              f"OpenMP over cells, {cores} threads")
    return {"value": cells * steps / el / 1e6, "unit": "MLUPS", "cores": cores, "kind": kind, "sample": sample,
            "ms_per_step": el / steps * 1e3}


def cpu_baseline(p, budget_s=25.0):
    """The reference's CPU path timed beside the B200 arm (time_reference_cpu,
    bounded to ~25 s): 3 warm-up and 20 timed steps, the sample the reference
    arm takes at the driver's step count."""
    r = time_reference_cpu(p, steps=20, warmup=3, budget_s=budget_s)
    r.pop("ms_per_step")
    return r


def reference_cuda(p, steps=20, warmup=3):
    """The reference's own CUDA build (oracle/_ref/ref_cuda_bench_{f64,f32}: its
    16 kernel files for sm_100a with --use_fast_math, driven through main.cpp's
    loop) on the same workload; a reported baseline, not the product."""
    import json as _json

    import numpy as np

    out = {}
    exes = {prec: os.path.join(ROOT, "oracle", "_ref", f"ref_cuda_bench_{prec}") for prec in ("f64", "f32")}
    if not all(os.path.exists(e) for e in exes.values()):
        return {"unavailable": "oracle/_ref/ref_cuda_bench_* not built (python oracle/build_oracle.py --cuda)"}
    if p.collision != "bgk" or p.isotherm not in ("langmuir", "linear"):
        return {"unavailable": "driver covers the BGK channel / pack set-up only"}
    iso = (p.q_max, p.b_langmuir, p.k_ldf) if p.isotherm == "langmuir" else (p.k_henry, 0.0, p.k_a)
    tau_ad = float(p.tau_ad) if np.isscalar(p.tau_ad) else float(np.asarray(p.tau_ad).reshape(-1)[0])
    with tempfile.TemporaryDirectory() as d:
        mask = os.path.join(d, "mask.bin")
        p.solid.astype(np.uint8).tofile(mask)
        for prec, exe in exes.items():
            args = [exe, mask, str(p.nx), str(p.ny), str(p.nz), str(steps), str(warmup), "bgk", p.isotherm,
                    repr(p.tau), repr(tau_ad), repr(p.u_in[0]), *[repr(float(v)) for v in iso]]
            r = subprocess.run(args, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, timeout=600)
            if r.returncode != 0:
                out[prec] = {"unavailable": r.stdout.strip().splitlines()[-1] if r.stdout.strip() else "failed"}
                continue
            line = _json.loads(r.stdout.strip().splitlines()[-1])
            out[prec] = {"value": line["mlups"], "unit": "MLUPS", "ms_per_step": line["ms_per_step"],
                         "steps": steps, "warmup": warmup}
    out["note"] = ("reference CUDA build (all 16 src/**/*.cu, --use_fast_math, -rdc, sm_100a), "
                   "same geometry and parameters, CUDA events around the steps")
    return out


def run_reference_arm(args, world, rank):
    if rank != 0:
        return
    p = make_problem(args)
    # warmup + steps take about two minutes
    r = time_reference_cpu(p, args.steps, args.warmup, 120.0)
    value = r["value"]
    line = {"impl": "reference", "metric": "coupled NS+AD MLUPS", "value": value, "unit": "MLUPS",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_desc(p),
            "cpu_baseline": {"value": value, "unit": "MLUPS", "cores": r["cores"], "kind": r["kind"],
                             "sample": r["sample"]},
            "e2e": {"value": value, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_sharded(args, p, world, rank, local, stream, barrier, max_over_ranks):
    """The one lattice cut into `world` z-slabs, one per GPU: every step updates
    each slab's boundary planes, sends their halos (the 6 crossing populations
    of a plane per inner face, NCCL point-to-point) while the interior planes
    update, then unpacks the received halos.  Total work is fixed: strong
    scaling."""
    import torch

    from fluidmaxxer_b200 import slabs

    L, sr = slabs.lattice_rank(p, rank, world, args.precision, stream=stream.cuda_stream)
    for _ in range(args.warmup):
        sr.step()
    torch.cuda.synchronize()
    vis = [v for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
    clocks = Clocks(vis[local].strip() if local < len(vis) else local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        sr.step()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    el_ms = max_over_ranks(e0.elapsed_time(e1))
    bt = sr.breakthrough(L.breakthrough(), device="cuda")     # the whole lattice's C_out(t)
    s = sr.slab
    part = np.empty(3)
    slabs.check(L._lib.fm_reduce_zrange(L.h, s.first, s.last + 1, part.ctypes.data))
    sums = sr.reduce(part, device="cuda")
    L.close()
    n = p.n_cells
    peak, peak_kind = measured_peak()
    bpc = BYTES_PER_CELL[args.precision]
    # per GPU: its own cells' algorithmic bytes over the whole step time
    achieved = bpc * (n / world) * args.steps / (el_ms / 1e3) / 1e9
    halo = sr.io.nbytes
    return {
        "metric": "coupled NS+AD MLUPS", "value": n * args.steps / (el_ms / 1e3) / 1e6, "unit": "MLUPS",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": el_ms / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": args.precision,
        "data": "synthetic",
        "config": dict(workload_desc(p), parallelism=f"z-slabs{world}", precision=args.precision),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind, "traffic": None, "algorithmic_bytes_per_cell": bpc,
                     "kernel": "the whole slab step per GPU (3 launches, halo pack / unpack, NCCL)"},
        "halo_bytes_per_step_per_inner_face_and_direction": halo,
        "c_out_final": float(bt[-1]) if len(bt) else None, "domain_sums": [float(v) for v in sums],
        "gpu_launches": args.steps * (3 + 2 * 2),   # 3 plane launches + pack/unpack per side, per rank
        "clocks": clk,
    }


def run_adjoint(args, world, rank, stream, barrier, max_over_ranks):
    """The differentiation form on its 128x64x64 smooth porous problem (porous
    BGK, Langmuir 4 / 1.0 / 0.03 against the curve of 5 / 1.3 / 0.04, C_out every
    20 steps over 4000 steps, checkpoints every 200, FP32): one "step" is one
    gradient evaluation (forward with checkpoints + reverse sweep).  value =
    cell-steps of the differentiated run per second of the whole evaluation."""
    import numpy as np
    import torch

    from fluidmaxxer_b200 import lattice, problems
    from fluidmaxxer_b200.adjoint import _set_parameters

    p = problems.smooth_porous()
    n_s = p.notes["n_s"]
    prec = args.precision if args.precision in ("f32", "f64") else "f32"
    L = lattice.from_problem(p, prec, stream=stream.cuda_stream)
    params = np.array([p.q_max, p.b_langmuir, p.k_ldf])
    _set_parameters(L, p, np.array([5.0, 1.3, 0.04]), n_s)
    L.step(p.steps)
    target = L.breakthrough()[1:]
    torch.cuda.synchronize()
    # forward only, the same steps (reference point)
    _set_parameters(L, p, params, n_s)
    f0 = torch.cuda.Event(enable_timing=True); f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream); L.step(p.steps); f1.record(stream)
    torch.cuda.synchronize()
    fwd_ms = f0.elapsed_time(f1)

    def grad_eval():
        _set_parameters(L, p, params, n_s)
        return L.adjoint_breakthrough(p.steps, target, checkpoint_every=200)

    for _ in range(max(args.warmup, 1)):
        grad_eval()
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        loss, gp, _ = grad_eval()
    torch.cuda.synchronize()
    el = max_over_ranks(time.perf_counter() - t0)
    recomputed, ws = L.adjoint_stats()
    L.close()
    ms = el * 1e3 / args.steps
    n = p.n_cells
    return {
        "metric": "adjoint cell-steps per second (MLUPS of the differentiated run)", "impl": "b200",
        "value": n * p.steps * world / (ms / 1e3) / 1e6, "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 1), "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": prec, "data": "synthetic",
        "config": {"workload": "smooth_porous_128x64x64 gradient", "cells": n, "forward_steps": p.steps,
                   "sample_every": p.sample_every, "checkpoint_every": 200, "isotherm": "langmuir",
                   "collision": "porous", "parallelism": "replicas" if world > 1 else "single",
                   "l2": "the state (58.7 MB) fits L2; host-timed whole evaluations (allocation-free after the first)"},
        "forward_ms": fwd_ms, "gradient_over_forward": ms / fwd_ms, "recomputed_steps": recomputed,
        "workspace_bytes": ws, "loss": loss, "grad_params": [float(v) for v in gp],
    }


def run_batch(args, world, rank, stream, barrier, max_over_ranks):
    """64 uneven porous samples (edges from {96..160}^3, Langmuir parameters
    drawn per sample) advanced together by the batch's replayed step graph.
    With --shard on N > 1 GPUs the samples are split across the ranks by cell
    count (independent samples: no exchange) and the value is all samples' cell
    updates over the slowest rank's time (strong scaling); otherwise every rank
    runs all samples (replicas, weak scaling)."""
    import torch

    from fluidmaxxer_b200 import lattice, problems
    all_ps = problems.batch_samples(count=args.samples)
    sharded = args.shard and world > 1
    if sharded:
        mine = lattice.partition_samples([p.n_cells for p in all_ps], world)[rank]
        ps = [all_ps[i] for i in mine]
    else:
        ps = all_ps
    cells = sum(p.n_cells for p in ps)
    total_cells = sum(p.n_cells for p in all_ps) if sharded else cells * world
    t0 = time.perf_counter()
    lats = [lattice.from_problem(p, args.precision, stream=stream.cuda_stream) for p in ps]
    B = lattice.Batch(lats, stream=stream.cuda_stream)
    setup_s = time.perf_counter() - t0
    cfg = B.autotune(trial_steps=4)
    B.step(args.warmup)
    torch.cuda.synchronize()
    barrier()
    clocks = Clocks(0)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    B.step(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    el_ms = max_over_ranks(e0.elapsed_time(e1))
    bt = [L.breakthrough() for L in lats]
    # the same samples stepped one lattice at a time (one launch per sample per
    # step), over as many steps as the batch
    torch.cuda.synchronize()
    s0 = torch.cuda.Event(enable_timing=True)
    s1 = torch.cuda.Event(enable_timing=True)
    k = args.steps
    s0.record(stream)
    for _ in range(k):
        for L in lats:
            L.step(1)
    s1.record(stream)
    torch.cuda.synchronize()
    solo_ms = s0.elapsed_time(s1)
    B.close()
    for L in lats:
        L.close()
    value = total_cells * args.steps / (el_ms / 1e3) / 1e6
    peak, peak_kind = measured_peak()
    bpc = BYTES_PER_CELL[args.precision]
    achieved = bpc * cells * args.steps / (el_ms / 1e3) / 1e9
    sizes = sorted({(p.nx, p.ny, p.nz) for p in all_ps})
    return {
        "metric": "coupled NS+AD MLUPS", "value": value, "unit": "MLUPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": el_ms / args.steps,
        "higher_is_better": True, "scaling": "strong" if sharded else "weak", "vs_baseline": None,
        "dtype": args.precision, "data": "synthetic",
        "config": {"workload": f"batch of {len(all_ps)} samples", "cells": sum(p.n_cells for p in all_ps),
                   "cells_this_rank": cells, "distinct_sizes": len(sizes),
                   "collision": "bgk", "isotherm": "langmuir (per-sample q_max, K_L, k_ads)",
                   "tau_ns": 0.7, "tau_ad": 0.6, "inlet_u": 0.01,
                   "l2": "each step streams ~29 GB (> 126 MB L2); no flush needed",
                   "autotuned": cfg,
                   "parallelism": f"samples{world}" if sharded else ("replicas" if world > 1 else "single")},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind, "traffic": None, "algorithmic_bytes_per_cell": bpc,
                     "kernel": ("k_coupled_step per sample in the batch graph" if cfg["mode"] == 3
                                else "k_coupled_batch") + " (whole step incl. probe launches)"},
        "per_sample_launches": {"value": cells * k / (solo_ms / 1e3) / 1e6, "unit": "MLUPS",
                                "note": "same samples, one fm_step launch per sample per step"},
        "gpu_launches": args.steps * (len(lats) if cfg["mode"] == 3 else 1)
        + (args.steps // 20) * (1 if any(len(b) for b in bt) else 0),
        "setup_s": setup_s, "breakthrough_samples_per_sample": int(len(bt[0])),
        "clocks": clk,
    }


def time_form(p, prec, args, stream, max_over_ranks, f32_value, peak, peak_kind, world):
    """One storage form on the bench workload: MLUPS over the timed steps, the
    fused kernel's mean launch time (CUDA events around every launch) and its
    HBM-roofline fraction at the form's algorithmic bytes per cell, and the
    copy ceiling of the form's own access pattern (fm_bench_pull_copy; for the
    16-bit forms in the pair layout, 32-bit words of two cells)."""
    import torch

    from fluidmaxxer_b200 import lattice
    n = p.n_cells
    Lp = lattice.from_problem(p, prec, stream=stream.cuda_stream)
    layout = Lp.storage_layout()
    kernel = {"pair-staged": "k_pair_staged", "pair": "k_coupled_pair"}.get(Lp.step_kernel(), "k_coupled_step")
    Lp.step(args.warmup)
    torch.cuda.synchronize()
    Lp.profile_enable(True)
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    Lp.step(args.steps)
    f1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(f0.elapsed_time(f1))
    kern_ms, launches = Lp.profile_read()
    kern_ms = max_over_ranks(kern_ms)
    pc_ms, pc_bytes = Lp.bench_pull_copy(20)
    pc_ms = max_over_ranks(pc_ms)
    Lp.close()
    mlups = n * args.steps * world / (ms / 1e3) / 1e6
    per_launch = kern_ms / max(launches, 1)
    bpc = BYTES_PER_CELL[prec]
    achieved = bpc * n / (per_launch / 1e3) / 1e9 if per_launch > 0 else 0.0
    pc_gbs = pc_bytes / (pc_ms / 1e3) / 1e9
    out = {"value": mlups, "unit": "MLUPS", "speedup_vs_f32": mlups / f32_value, "layout": layout,
           "kernel": kernel,
           "kernel_ms_per_launch": per_launch,
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                        "peak_source": peak_kind, "algorithmic_bytes_per_cell": bpc},
           "pattern_copy": {"achieved": pc_gbs, "unit": "GB/s", "frac": pc_gbs / peak,
                            "step_vs_pattern": achieved / pc_gbs if pc_gbs > 0 else None,
                            "ceiling_vs_f32_mlups": (pc_gbs * 1e3 / (2 * BYTES_PER_POP[prec] * 26)) / f32_value}}
    if prec in ("f16", "bf16", "f16q"):
        out["pair_layout"] = time_pair_kernels(p, prec, args, stream, max_over_ranks, peak)
    return out


def time_pair_kernels(p, prec, args, stream, max_over_ranks, peak):
    """The opt-in pair layout of a 16-bit form (two cells per 32-bit word):
    kernel time per launch of k_coupled_pair and of the staged kernel, and
    the copy ceiling of the pair access pattern, over min(steps, 200) steps
    after the warm-up -- beside the default one-cell kernel they lose to."""
    import torch

    from fluidmaxxer_b200 import lattice
    res = {}
    steps = min(args.steps, 200)
    for name, staged in (("k_pair_staged", True), ("k_coupled_pair", False)):
        L = lattice.from_problem(p, prec, stream=stream.cuda_stream)
        L.set_pair_layout(True)
        L.set_pair_kernel(staged)
        L.step(args.warmup)
        torch.cuda.synchronize()
        L.profile_enable(True)
        L.step(steps)
        torch.cuda.synchronize()
        kern_ms, launches = L.profile_read()
        per = max_over_ranks(kern_ms) / max(launches, 1)
        res[name] = {"kernel_ms_per_launch": per, "steps": steps,
                     "hbm_frac": BYTES_PER_CELL[prec] * p.n_cells / (per / 1e3) / 1e9 / peak}
        if not staged:
            pc_ms, pc_bytes = L.bench_pull_copy(20)
            pc_gbs = pc_bytes / (max_over_ranks(pc_ms) / 1e3) / 1e9
            res["pattern_copy"] = {"achieved": pc_gbs, "unit": "GB/s", "frac": pc_gbs / peak}
        L.close()
    return res


def time_batch_form(args, stream, max_over_ranks, f32_value, peak, peak_kind, world, samples=64):
    """The batching form on its own workload (64 uneven porous samples, edges
    from {96..160}^3, per-sample Langmuir parameters, FP32), autotuned, timed
    over the bench's step count after its warm-up; roofline at 216 B per cell."""
    import torch

    from fluidmaxxer_b200 import lattice, problems
    ps = problems.batch_samples(count=samples)
    cells = sum(q.n_cells for q in ps)
    lats = [lattice.from_problem(q, "f32", stream=stream.cuda_stream) for q in ps]
    B = lattice.Batch(lats, stream=stream.cuda_stream)
    cfg = B.autotune(trial_steps=4)
    B.step(args.warmup)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    B.step(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1))
    B.close()
    for L in lats:
        L.close()
    mlups = cells * args.steps * world / (ms / 1e3) / 1e6
    achieved = BYTES_PER_CELL["f32"] * cells * args.steps / (ms / 1e3) / 1e9
    return {"value": mlups, "unit": "MLUPS", "workload": f"batch of {samples} samples, {cells} cells",
            "autotuned": cfg, "ms_per_step": ms / args.steps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": peak_kind, "algorithmic_bytes_per_cell": BYTES_PER_CELL["f32"],
                         "kernel": "the whole batch step (all launches and probes)"}}


def max_over_ranks_of(v, world, device):
    """Max of a per-rank float over the process group (the timing rule: the
    slowest replica sets the job's time); the only collective of the data path
    besides the barriers, since every rank steps its own lattice."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_mlups(cells_per_rank, steps, world, max_ms):
    """Whole-job throughput of N replicas: all ranks' cell updates over the
    slowest rank's time (weak scaling, per-GPU work fixed)."""
    return cells_per_rank * steps * world / (max_ms / 1e3) / 1e6


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, world, rank)
        return

    import torch
    import torch.distributed as dist
    from datetime import timedelta

    from fluidmaxxer_b200 import lattice
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(v):
        return max_over_ranks_of(v, world, "cuda")

    if args.workload == "adjoint":
        stream = torch.cuda.Stream()
        torch.cuda.set_stream(stream)
        line = run_adjoint(args, world, rank, stream, barrier, max_over_ranks)
        if rank == 0:
            print(json.dumps(line), flush=True)
        if world > 1:
            dist.destroy_process_group()
        return
    if args.workload == "batch":
        stream = torch.cuda.Stream()
        torch.cuda.set_stream(stream)
        line = run_batch(args, world, rank, stream, barrier, max_over_ranks)
        if rank == 0:
            print(json.dumps(line), flush=True)
        if world > 1:
            dist.destroy_process_group()
        return

    p = make_problem(args)
    # a dedicated stream: the lattice queues its kernels on it and the events
    # below are recorded on it (the legacy default stream would not order with
    # a library-owned non-blocking stream)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    if args.shard and world > 1:
        line = run_sharded(args, p, world, rank, local, stream, barrier, max_over_ranks)
        if rank == 0:
            print(json.dumps(line), flush=True)
        dist.destroy_process_group()
        return

    L = lattice.from_problem(p, args.precision, stream=stream.cuda_stream)
    if args.prefetch is not None:
        L.set_prefetch_distance(args.prefetch)
    if args.pair_kernel != "off":
        L.set_pair_layout(True)
        L.set_pair_kernel(args.pair_kernel == "staged")
    main_kernel = {"pair-staged": "k_pair_staged", "pair": "k_coupled_pair"}.get(L.step_kernel(), "k_coupled_step")
    L.step(args.warmup)
    torch.cuda.synchronize()

    vis = [v for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
    clocks = Clocks(vis[local].strip() if local < len(vis) else local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    L.profile_enable(True)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    L.step(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    el_ms = max_over_ranks(e0.elapsed_time(e1))
    kern_ms, launches = L.profile_read()
    kern_ms = max_over_ranks(kern_ms)
    launches_per_step = L.launches_per_step()
    # the same access pattern as a pure copy (no arithmetic): the ceiling of
    # the pulls and stores themselves, after the timed region
    pc_ms, pc_bytes = L.bench_pull_copy(20)
    pc_ms = max_over_ranks(pc_ms)
    L.close()

    n = p.n_cells
    value = job_mlups(n, args.steps, world, el_ms)
    peak, peak_kind = measured_peak()
    bpc = BYTES_PER_CELL[args.precision]
    achieved = bpc * n * launches / (kern_ms / 1e3) / 1e9 if kern_ms > 0 else 0.0
    tpc = traffic_per_cell(args.precision) if main_kernel == "k_coupled_step" else None
    line = {
        "metric": "coupled NS+AD MLUPS", "value": value, "unit": "MLUPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": el_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": args.precision, "data": "synthetic",
        "config": dict(workload_desc(p), parallelism="replicas" if world > 1 else "single",
                       precision=args.precision),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "traffic": None if tpc is None else tpc * n,
                     "algorithmic_bytes_per_cell": bpc, "kernel": main_kernel,
                     "kernel_ms_per_launch": kern_ms / max(launches, 1),
                     "pattern_copy": {"achieved": pc_bytes / (pc_ms / 1e3) / 1e9, "unit": "GB/s",
                                      "frac": pc_bytes / (pc_ms / 1e3) / 1e9 / peak,
                                      "step_vs_pattern": achieved / (pc_bytes / (pc_ms / 1e3) / 1e9),
                                      "what": "k_pull_copy: the step's 26 pulls and 26 stores per cell as a "
                                              "pure copy (fm_bench_pull_copy), 20 launches after the timed region"}},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clk,
    }

    if not args.no_e2e:
        # the caller's result buffers, page-locked, allocated before the timed
        # region, in the form's arithmetic type (FP32 for every form but FP64,
        # as the reference's FP32 build downloads its DATA_TYPE fields)
        fdt = np.float64 if args.precision == "f64" else np.float32
        tdt = torch.float64 if args.precision == "f64" else torch.float32
        pinned = {k: torch.empty(n, dtype=tdt, pin_memory=True).numpy()
                  for k in ("rho", "ux", "uy", "uz", "phi", "q")}
        # three whole jobs, the median reported (a single host-timed job is
        # exposed to one-off host or allocator stalls); the first is also
        # reported on its own
        runs, phases = [], []
        for _ in range(3):
            barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            L2 = lattice.from_problem(p, args.precision, stream=stream.cuda_stream)
            L2.synchronize()
            t1 = time.perf_counter()
            L2.step(args.steps)
            bt = L2.breakthrough()
            t2 = time.perf_counter()
            flds = L2.fields(out=pinned, dtype=fdt)
            t3 = time.perf_counter()
            L2.close()
            torch.cuda.synchronize()
            t4 = time.perf_counter()
            runs.append(max_over_ranks(t4 - t0))
            phases.append({"setup_ms": (t1 - t0) * 1e3, "steps_ms": (t2 - t1) * 1e3, "download_ms": (t3 - t2) * 1e3,
                           "destroy_ms": (t4 - t3) * 1e3})
        e2e_s = statistics.median(runs)
        h2d = 7 * n + (0 if np.isscalar(p.tau_ad) else 8 * n)   # seven byte masks (+ a float64 tau field)
        d2h = 6 * np.dtype(fdt).itemsize * n + 8 * len(bt)   # six fields + the breakthrough series
        mid = runs.index(sorted(runs)[1])
        line["e2e"] = {"value": n * args.steps * world / e2e_s / 1e6, "unit": "MLUPS",
                       "runs_mlups": [round(n * args.steps * world / r / 1e6, 1) for r in runs],
                       "first_job_mlups": round(n * args.steps * world / runs[0] / 1e6, 1),
                       "median_job_ms": {k: round(v, 2) for k, v in phases[mid].items()},
                       "fixed_ms": round((e2e_s - args.steps * (el_ms / args.steps) / 1e3) * 1e3, 1),
                       "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
                       "includes": "lattice create + geometry/field upload + init + steps + breakthrough "
                                   f"and 6 {np.dtype(fdt).name} field downloads into page-locked buffers + destroy, "
                                   "via the C ABI; median of 3 such jobs"}
        del flds

    if not args.no_forms and args.precision == "f32" and args.workload == "sphere_pack":
        forms = {}
        # the 16-bit storage forms, and FP64 (the reference's shipped DATA_TYPE)
        for prec in ("f16", "bf16", "f16q", "f64"):
            forms[prec] = time_form(p, prec, args, stream, max_over_ranks, value, peak, peak_kind, world)
        if not args.no_batch:
            forms["batch"] = time_batch_form(args, stream, max_over_ranks, value, peak, peak_kind, world)
        line["forms"] = forms

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(p)
    if rank == 0 and world == 1 and not args.no_reference_cuda:
        line["reference_cuda"] = reference_cuda(p)

    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
