"""Benchmark of the FastEddy hot path on B200: RK3 cell-updates/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--case NAME]

Workload (default): the moist convective boundary layer over a Gaussian hill,
512 x 512 x 128 cells, dx = dy = 20 m, dz = 10 m, terrain-following grid, prognostic
q_v and q_l with saturation adjustment, 1.5-order TKE, surface layer, Rayleigh damping.
Inputs are synthetic (seeded theta perturbations, analytic hill and q_v profile).

Our arm: a step is one RK3 step (3 fused stage kernels + the last-stage physics kernel)
replayed from a CUDA graph on the resident device state (8 fields, 1.15 GB, far larger
than the 126 MB L2, so no flush is needed between steps). `e2e` is the same metric
through the drop-in C ABI (cuda_timeIntCommence) with host buffers: upload of the host
state, K steps, copy-back of state, pressure and surface arrays inside the timed region.

Reference arm: the reference's own implementation of this path is CUDA-only; its code,
compiled for sm_100a from the reference sources (oracle/_ref), runs the same case
through its own cuda_timeIntCommence and is timed the same way.

Multi-GPU: the path does not shard (single-domain model, no halo exchange), so N GPUs run
N independent replicas; value is the whole-job rate, timed as the max over ranks.
"""
from __future__ import annotations

import argparse
import importlib
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CASES = {
    # name: (case key, Nx, Ny, Nz, hill, prognostic fields, description)
    "moist_hill_512": ("cbl_moist_hill", 512, 512, 128, True, 8,
                       "moist CBL over a Gaussian hill, 512x512x128, dx=dy=20 m, dz=10 m"),
    "moist_hill_256": ("cbl_moist_hill", 256, 256, 128, True, 8,
                       "moist CBL over a Gaussian hill, 256x256x128, dx=dy=20 m, dz=10 m"),
    "dry_cbl_128": ("cbl_dry", 128, 128, 64, False, 6, "dry CBL, flat, 128x128x64, dx=dy=20 m, dz=10 m"),
    "bomex_512": ("bomex", 512, 512, 128, False, 8,
                  "moist CBL with the BOMEX tutorial's selectors (HYB34 for q_v, explicit filter, large-scale "
                  "forcing with slab-mean subsidence), flat, 512x512x128, dx=dy=20 m, dz=10 m"),
    "dry_hill_1024": ("cbl_hill_dry", 1024, 1024, 256, True, 6,
                      "dry CBL over a Gaussian hill, 1024x1024x256, dx=dy=20 m, dz=10 m"),
}
DEFAULT_CASE = "moist_hill_512"
ENSEMBLE_CASE = "ensemble64"


def ensemble_specs(n: int = 64, seed: int = 2024) -> list[tuple[int, int, int, float, float]]:
    """Seeded member draws of the batched neutral-ABL ensemble: Nx, Ny in 64..192, Nz in 64..96,
    U_g uniform in 5..15 m/s, z0 log-uniform in 0.01..0.5 m."""
    import random

    rng = random.Random(seed)
    out = []
    for _ in range(n):
        nx, ny, nz = rng.randint(64, 192), rng.randint(64, 192), rng.randint(64, 96)
        ug = rng.uniform(5.0, 15.0)
        z0 = math.exp(rng.uniform(math.log(0.01), math.log(0.5)))
        out.append((nx, ny, nz, round(ug, 3), round(z0, 4)))
    return out


def case_text_module():
    """The parameter-file writer (fasteddy-model_b200/cases.py) loaded on its own: plain Python
    text generation, so the reference arm maps none of this repository's native libraries and
    imports nothing of its package."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("fe_case_text", os.path.join(ROOT, "fasteddy-model_b200", "cases.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def hill_topofile_bytes(nx: int, ny: int, dx: float, dy: float, height: float, halfwidth: float) -> bytes:
    """The Gaussian hill h = height * 2^-(r/halfwidth)^2 (r from cell centres to the domain
    centre) in the reference's topoFile format (grid.c:313-326): int Nx, int Ny, float[Ny][Nx]."""
    import numpy as np

    x = (np.arange(nx) + 0.5) * dx - 0.5 * nx * dx
    y = (np.arange(ny) + 0.5) * dy - 0.5 * ny * dy
    r = np.sqrt(x[:, None] ** 2 + y[None, :] ** 2) / halfwidth
    h = (height * np.power(2.0, -r * r)).astype(np.float32)  # [i][j]
    return np.array([nx, ny], np.int32).tobytes() + np.ascontiguousarray(h.T).tobytes()


def case_config(case: str, world: int) -> dict:
    """The `config` of a bench line: the workload only, identical in both arms."""
    key, nx, ny, nz, terrain, nprog, desc = CASES[case]
    text = case_text_module()
    return {"workload": desc, "cells": nx * ny * nz, "prognostic_fields": nprog, "dt_s": float(text.DT_STABLE),
            "parallelism": f"replicas{world}",
            "l2": f"state {4 * nprog * (nx + 6) * (ny + 6) * (nz + 6) / 1e9:.2f} GB per copy >> 126 MB L2, no flush needed"}


def graph_warmup(w: int) -> int:
    """Untimed warm-up steps: at least w, rounded up to whole 8-step graph batches, so that the
    engine's CUDA graph is captured and instantiated before the timed region."""
    return 8 * max(1, math.ceil(w / 8))


def bytes_per_cell_stage(nprog: int) -> int:
    """Algorithmic HBM bytes per cell of one RK stage kernel (the second stage): read phi and
    phi0 and write phi (3 N_p floats), read and write p' (2), and read the 8 per-cell grid and
    base-state fields every stage needs (D, 1/D, J31, J32, J33, z, rho_BS, p_BS)."""
    return 4 * (3 * nprog + 2 + 8)


# ---------------------------------------------------------------- distributed helpers
def dist_env() -> tuple[int, int, int]:
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def max_over_ranks(value: float, device: str = "cpu") -> float:
    """Max of a per-rank float over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return value
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(device: str = "cpu") -> None:
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def whole_job_rate(cells_per_rank: int, steps: int, max_seconds: float, world: int) -> float:
    """Cell-updates/s of the whole job: every rank advances its own replica."""
    return cells_per_rank * steps * world / max_seconds


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int) -> None:
        self.gpu = gpu_index
        self.lines: list[str] = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self) -> None:
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc) -> None:
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- roofline helpers
def measured_peak_gbs() -> tuple[float, str]:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            v = float(json.load(f)["hbm_gbs"])
        return v, "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def measured_peak_tflops() -> tuple[float, str]:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["bf16_tflops"]), "measured"
    except (OSError, KeyError, ValueError):
        return 1590.0, "fallback"


# tensor-core FLOPs the network kernels execute (tiles of 128 cells, padded widths 16/64/16)
MLP_FWD_FLOP = 2 * (16 * 64 + 64 * 64 + 64 * 64 + 64 * 16)              # per cell
MLP_TRAIN_FLOP = MLP_FWD_FLOP + 2 * (16 * 64 + 64 * 64 + 64 * 64) + 2 * 128 * (16 + 64 + 64 + 64)  # per sample


def measure_learned(fe, dom, args, cells: int, stream, local: int) -> dict:
    """The learned-SGS form of the same workload: the network (trained briefly on a strided
    sample of this run's own closure stresses, so its outputs have the right size; the cost
    does not depend on the weights) replaces the closure's stresses at every physics stage."""
    import torch

    m = fe.Mlp(device=local, seed=7)
    every = max(1, cells // 524288)
    s = dom.sgs_sample(every)
    m.set_data(s["X"], s["tau"] / s["rho"][:, None])
    nsamp = int(s["X"].shape[0])
    del s
    m.train(100, 4096, 2e-3)
    dom.set_sgs_mlp(m)
    dom.advance(graph_warmup(args.warmup))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    dom.advance(args.steps, sync=False)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    nonfinite = dom.nonfinite()
    dom.set_sgs_mlp(None)
    peak, src = measured_peak_tflops()
    inf_ms = m.time(False, nsamp, reps=10)
    trn_ms = m.time(True, nsamp, reps=5)
    m.close()
    inf_tf = MLP_FWD_FLOP * nsamp / (inf_ms * 1e-3) / 1e12
    trn_tf = MLP_TRAIN_FLOP * nsamp / (trn_ms * 1e-3) / 1e12
    return {
        "value": cells * args.steps / (ms * 1e-3), "unit": "cell-updates/s", "ms_per_step": ms / args.steps,
        "nonfinite_cells": nonfinite,
        "closure": "BF16 MLP 11-64-64-64-9 (tcgen05) replacing the TKE closure's 9 stresses at each physics stage",
        "mlp_inference": {"cells_per_s": nsamp / (inf_ms * 1e-3), "tflops": inf_tf, "peak_tflops": peak,
                          "frac": inf_tf / peak, "peak_source": src, "flop_per_cell": MLP_FWD_FLOP,
                          "sample": f"{nsamp} cells, inputs/outputs FP32 in HBM"},
        "mlp_training": {"samples_per_s": nsamp / (trn_ms * 1e-3), "tflops": trn_tf, "frac": trn_tf / peak,
                         "flop_per_sample": MLP_TRAIN_FLOP},
    }


def profiled_traffic(case: str) -> float | None:
    """DRAM bytes per launch of the stage kernel from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", f"k_march_{case}.txt")
    try:
        for line in open(p):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


# ---------------------------------------------------------------- CPU baseline
def cpu_baseline(fe, case_key: str, seconds_target: float = 8.0) -> dict:
    """The FP64 C restatement of the path (oracle), single thread, on a sample of the
    workload: the same case on a horizontal subdomain with the full column."""
    c = CASES[case_key]
    return cpu_baseline_case(fe, c[0], c[3], seconds_target)


def cpu_baseline_case(fe, case: str, nz: int, seconds_target: float = 8.0) -> dict:
    from oracle.pyoracle import Oracle

    n = 32
    host = fe.cases.setup_host(case, n, n, nz)
    o = Oracle(host.config())
    o.set_inputs(host.inputs())
    t0 = time.perf_counter()
    o.step(1)
    t1 = time.perf_counter()
    one = t1 - t0
    steps = max(1, int(seconds_target / max(one, 1e-3)) - 1)
    o.step(steps)
    t2 = time.perf_counter()
    o.close()
    host.cleanup()
    total_steps = steps + 1
    rate = n * n * nz * total_steps / (t2 - t0)
    return {"value": rate, "unit": "cell-updates/s", "cores": 1, "kind": "port",
            "sample": f"{total_steps} RK3 steps of the same case on a {n}x{n}x{nz} subdomain, "
                      f"serial FP64 C restatement ({t2 - t0:.1f} s)"}


# ---------------------------------------------------------------- our arm
def run_ours(args, rank: int, world: int, local: int) -> dict | None:
    import torch

    fe = importlib.import_module("fasteddy-model_b200")
    key, nx, ny, nz, terrain, nprog, desc = CASES[args.case]
    device = f"cuda:{local}"
    torch.cuda.set_device(local)
    host = fe.cases.setup_host(key, nx, ny, nz, seed=12345 + rank)
    inp = host.inputs()
    cfg = host.config()
    dom = fe.Domain(cfg, device=local)
    dom.set_inputs(inp)
    if args.autotune:
        dom.autotune()
    cells = nx * ny * nz
    warm = graph_warmup(args.warmup)
    dom.advance(warm)
    shape = list(dom.stage_kernel())  # form, rows per tile, planes per block
    stream = torch.cuda.ExternalStream(dom.stream(), device=device)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    l0 = dom.launch_count()
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        e0.record(stream)
        dom.advance(args.steps, sync=False)
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize()
    barrier()
    launches = dom.launch_count() - l0
    ms = e0.elapsed_time(e1)
    max_ms = max_over_ranks(ms, device)
    value = whole_job_rate(cells, args.steps, max_ms / 1e3, world)
    # dominant kernel: the fused dynamics stage, timed alone with CUDA events
    stage_ms = dom.time_stage_kernel(reps=10)
    bpc = bytes_per_cell_stage(nprog)
    achieved = bpc * cells / (stage_ms * 1e-3) / 1e9
    peak, peak_src = measured_peak_gbs()
    traffic = profiled_traffic(args.case)
    nonfinite = dom.nonfinite()
    learned = measure_learned(fe, dom, args, cells, stream, local) if (cfg.turbulenceSelector and not args.no_learned) else None
    dom.close()
    # end to end through the drop-in C ABI with host buffers
    libs = fe.load()
    ra = libs["refabi"]
    host.set_gi("NtBatch", args.steps)
    for fn in ("fecuda_Init", "cuda_gridInit", "cuda_hydroCoreInit", "cuda_timeIntInit"):
        rc = getattr(ra, fn)()
        if rc:
            raise RuntimeError(f"{fn} failed ({rc}): {libs['engine'].fe_last_error().decode()}")
    ra.cuda_timeIntCommence(host.gi("simTime_itRestart"))  # warm-up batch (graph capture)
    host.set_gi("simTime_it", 0)
    barrier()
    t0 = time.perf_counter()
    rc = ra.cuda_timeIntCommence(host.gi("simTime_itRestart"))  # uploads host state, K steps, copies back
    t1 = time.perf_counter()
    barrier()
    if rc:
        raise RuntimeError(f"cuda_timeIntCommence failed ({rc})")
    e2e_s = max_over_ranks(t1 - t0, device)
    ra.cuda_hydroCoreCleanup()
    n3 = (nx + 6) * (ny + 6) * (nz + 6)
    n2 = (nx + 6) * (ny + 6)
    nm = cfg.moistureNvars if cfg.moistureSelector else 0
    ntke = 1 if cfg.TKESelector else 0
    h2d = 4 * (n3 * (5 + ntke + nm) + n2 * (7 if nm else 5))
    d2h = 4 * (n3 * (5 + ntke + nm + 1) + n2 * (6 if nm else 4))
    clocks = clk.summary()
    host.cleanup()
    if rank != 0:
        return None
    line = {
        "metric": "RK3 cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": case_config(args.case, world),
        "warmup_steps_run": warm, "stage_kernel": shape,
        "e2e": {"value": whole_job_rate(cells, args.steps, e2e_s, world), "unit": "cell-updates/s",
                "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
                "path": "cuda_timeIntCommence (drop-in C ABI), host buffers, one batch of K steps"},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "kernel": "k_march (fused tendency + RK3 commit, stage 2 of 3)", "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "peak_source": peak_src, "bytes_per_cell_stage": bpc, "stage_kernel_ms": stage_ms},
        "clocks": clocks,
        "nonfinite_cells": nonfinite,
    }
    if learned is not None:
        line["learned_sgs"] = learned
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(fe, args.case)
    return line


# ---------------------------------------------------------------- batched ensemble
def run_ensemble(args, rank: int, world: int, local: int) -> dict | None:
    """64 uneven neutral-ABL members advanced together in one captured CUDA graph per 8 steps:
    each step is one work-list launch per kernel over the tiles of all members (the members'
    parameters in device tables), or, with --ensemble-branches, one graph branch per member."""
    import numpy as np
    import torch

    fe = importlib.import_module("fasteddy-model_b200")
    device = f"cuda:{local}"
    torch.cuda.set_device(local)
    specs = ensemble_specs()
    doms, inputs, shapes = [], [], []
    t_tune = time.perf_counter()
    for i, (nx, ny, nz, ug, z0) in enumerate(specs):
        host = fe.cases.setup_host("abl_neutral", nx, ny, nz, seed=1000 + i + 97 * rank, ug=ug, z0=z0)
        inp, cfg = host.inputs(), host.config()
        host.cleanup()
        d = fe.Domain(cfg, device=local)
        d.set_inputs(inp)
        d.autotune()
        doms.append(d)
        inputs.append(inp)
        shapes.append(d.stage_kernel())
    t_tune = time.perf_counter() - t_tune
    cells = sum(nx * ny * nz for nx, ny, nz, _, _ in specs)
    ens = fe.Ensemble(doms)
    ens.set_batched(not args.ensemble_branches)
    ens.advance(graph_warmup(args.warmup))
    stream = torch.cuda.ExternalStream(ens.stream(), device=device)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    steps = 8 * max(1, math.ceil(args.steps / 8))
    launches0 = ens.launch_count()
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        e0.record(stream)
        ens.advance(steps, sync=False)
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    launches = ens.launch_count() - launches0
    form = "work list: one launch per kernel of a step over the tiles of all members" if ens.batched() else \
        "one CUDA-graph branch per member"
    max_ms = max_over_ranks(ms, device)
    value = whole_job_rate(cells, steps, max_ms / 1e3, world)
    # stage kernels of every member, timed alone: algorithmic bytes over summed launch times
    bpc = bytes_per_cell_stage(6)
    stage_ms = sum(d.time_stage_kernel(reps=5) for d in doms)
    achieved = bpc * cells / (stage_ms * 1e-3) / 1e9
    peak, peak_src = measured_peak_gbs()
    nonfinite = sum(d.nonfinite() for d in doms)
    # end to end through the public API: upload every member's host state, K steps, download;
    # the host arrays are page-locked once beforehand, as a host that keeps its state does
    outs = [d.state_buffers() for d in doms]
    pinned = [a for inp in inputs for a in (inp["hydroFlds"], inp.get("sgstke"))] + \
             [a for o in outs for a in o.values()]
    for a in pinned:
        fe.runtime.pin(a)
    barrier()
    t0 = time.perf_counter()
    for d, inp in zip(doms, inputs):
        d.set_state(inp["hydroFlds"], inp.get("sgstke"), inp.get("moist"))
    ens.advance(steps)
    for d, o in zip(doms, outs):
        d.get_state(out=o)
    t1 = time.perf_counter()
    barrier()
    for a in pinned:
        fe.runtime.unpin(a)
    e2e_s = max_over_ranks(t1 - t0, device)
    h2d = sum(inp["hydroFlds"].nbytes + (inp["sgstke"].nbytes if inp.get("sgstke") is not None else 0) for inp in inputs)
    d2h = sum(sum(v.nbytes for v in o.values() if v is not None) for o in outs)
    ens.close()
    for d in doms:
        d.close()
    if rank != 0:
        return None
    kinds = {}
    for k, tj, ni in shapes:
        key = f"{k}:{tj}x{ni}"
        kinds[key] = kinds.get(key, 0) + 1
    line = {
        "metric": "RK3 cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": steps,
        "warmup": graph_warmup(args.warmup), "ms_per_step": max_ms / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "batched ensemble of 64 neutral ABL members, Nx,Ny in 64..192, Nz in 64..96, "
                               "U_g 5..15 m/s, z0 0.01..0.5 m (seeded), dx=dy=20 m, dz=10 m",
                   "members": len(specs), "cells": cells, "parallelism": f"replicas{world}",
                   "l2": f"state of all members {4 * 6 * cells / 1e9:.1f} GB >> 126 MB L2, no flush needed",
                   "autotuned_shapes": kinds, "autotune_s": round(t_tune, 1), "launch_form": form},
        "e2e": {"value": whole_job_rate(cells, steps, e2e_s, world), "unit": "cell-updates/s",
                "h2d_bytes_per_step": h2d / steps, "d2h_bytes_per_step": d2h / steps,
                "path": "engine API: fe_set_state of every member, one ensemble advance, fe_get_state "
                        "(page-locked host arrays)"},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "kernel": "k_march (all members, summed)", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "traffic": None, "peak_source": peak_src,
                     "bytes_per_cell_stage": bpc, "stage_kernel_ms_sum": stage_ms},
        "clocks": clk.summary(),
        "nonfinite_cells": nonfinite,
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_case(fe, "abl_neutral", 80)
    return line


# ---------------------------------------------------------------- the other configurations
def other_configs(args, local: int) -> dict:
    """The batched ensemble and the 1024x1024x256 domain (plain and learned closure), measured in
    the same one-GPU process after the headline case, each with its own device-timed rate and its
    end-to-end rate; their full lines come from --case ensemble64 / --case dry_hill_1024."""
    out = {}
    sub = argparse.Namespace(**vars(args))
    sub.no_cpu_baseline = True
    sub.case, sub.steps, sub.warmup = ENSEMBLE_CASE, 16, max(3, args.warmup)
    e = run_ensemble(sub, 0, 1, local)
    out[ENSEMBLE_CASE] = {"workload": e["config"]["workload"], "value": e["value"], "ms_per_step": e["ms_per_step"],
                          "steps": e["steps"], "e2e": e["e2e"]["value"], "gpu_launches": e["gpu_launches"],
                          "nonfinite_cells": e["nonfinite_cells"]}
    sub.case, sub.steps, sub.warmup, sub.no_learned = "dry_hill_1024", 5, 3, False
    r = run_ours(sub, 0, 1, local)
    big = {"workload": r["config"]["workload"], "value": r["value"], "ms_per_step": r["ms_per_step"],
           "steps": r["steps"], "e2e": r["e2e"]["value"], "roofline_frac": r["roofline"]["frac"],
           "nonfinite_cells": r["nonfinite_cells"]}
    if "learned_sgs" in r:
        big["learned_ms_per_step"] = r["learned_sgs"]["ms_per_step"]
        big["learned_value"] = r["learned_sgs"]["value"]
    out["dry_hill_1024"] = big
    return out


# ---------------------------------------------------------------- reference arm
def run_reference(args, rank: int, world: int) -> dict | None:
    """The reference's own CUDA build (oracle/_ref/fe_ref_harness, compiled from the reference
    sources for sm_100a) on the same case through its own cuda_timeIntCommence, from its own
    initial state: its grid from the case's topoFile, its base state and its theta
    perturbations; the reference cannot start moisture without a netCDF file, so the harness
    sets the case's q_v profile in C. Nothing of this repository's package or native libraries
    is loaded here. Only rank 0 runs it (a single process)."""
    if rank != 0:
        return None
    if args.case == ENSEMBLE_CASE:
        return run_reference_ensemble(args, world)
    key, nx, ny, nz, terrain, nprog, desc = CASES[args.case]
    base = {"metric": "RK3 cell-updates/s", "unit": "cell-updates/s", "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": case_config(args.case, 1)}
    try:
        from oracle import refrun
        if not refrun.available():
            from oracle import build_ref
            build_ref.build()
        text_mod = case_text_module()
        files, topo = {}, ""
        if terrain:
            files["hill.topo"] = hill_topofile_bytes(nx, ny, 20.0, 20.0, text_mod.HILL_HEIGHT, text_mod.HILL_HALFWIDTH)
            topo = "./hill.topo"
        text = text_mod.param_text(key, nx, ny, nz, topo=topo)
        qv = None
        if key in ("cbl_moist_hill", "bomex"):
            qv = "qv:%g,%g,%g" % (text_mod.QV_SFC, text_mod.QV_TOP, text_mod.QV_ZTOP)
        with ClockSampler(0) as clk:
            t = refrun.time_steps(text, None, args.steps, qv=qv, files=files)
    except Exception as exc:  # the reference cannot run here: report why
        return {"impl": "reference", "unavailable": f"{type(exc).__name__}: {str(exc).splitlines()[0][:200]}"}
    ms = t["ms_per_step"]
    value = nx * ny * nz / (ms * 1e-3)
    base.update({
        "value": value, "ms_per_step": ms,
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": 0, "kind": "reference",
                         "sample": f"reference CUDA build (oracle/_ref, sm_100a) on the B200 through its own "
                                   f"cuda_timeIntCommence, its own initial state: ({2 * args.steps}-step batch - "
                                   f"{args.steps}-step batch)/{args.steps}; the reference has no CPU implementation "
                                   f"of this path"},
        "clocks": clk.summary(),
        "reference_timing": t,
    })
    return base


def run_reference_ensemble(args, world: int) -> dict:
    """The reference has no ensemble launcher: its baseline for the 64 members is 64 sequential
    runs of its own build, one member per process, each timed as (2K-step batch - K-step batch)/K
    through its own cuda_timeIntCommence; the job's time per step is the sum over the members."""
    base = {"metric": "RK3 cell-updates/s", "unit": "cell-updates/s", "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic"}
    try:
        from oracle import refrun
        if not refrun.available():
            from oracle import build_ref
            build_ref.build()
        text_mod = case_text_module()
        specs = ensemble_specs()
        total_ms, cells = 0.0, 0
        with ClockSampler(0) as clk:
            for nx, ny, nz, ug, z0 in specs:
                # the tutorials' thread-block shape, as for the single-domain cases (the reference's
                # grid rounds up, so it covers these uneven sizes)
                text = text_mod.param_text("abl_neutral", nx, ny, nz, ug=ug, z0=z0)
                t = refrun.time_steps(text, None, args.steps)
                total_ms += t["ms_per_step"]
                cells += nx * ny * nz
    except Exception as exc:  # the reference cannot run here: report why
        return {"impl": "reference", "unavailable": f"{type(exc).__name__}: {str(exc).splitlines()[0][:200]}"}
    value = cells / (total_ms * 1e-3)
    base.update({
        "value": value, "ms_per_step": total_ms,
        "config": {"workload": "batched ensemble of 64 neutral ABL members, Nx,Ny in 64..192, Nz in 64..96, "
                               "U_g 5..15 m/s, z0 0.01..0.5 m (seeded), dx=dy=20 m, dz=10 m",
                   "members": len(specs), "cells": cells, "parallelism": f"replicas{world}"},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": 0, "kind": "reference",
                         "sample": "64 sequential runs of the reference CUDA build (oracle/_ref, sm_100a), one "
                                   "member each, per-step times summed; the reference has no CPU implementation "
                                   "of this path"},
        "clocks": clk.summary(),
    })
    return base


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--case", choices=sorted(CASES) + [ENSEMBLE_CASE], default=DEFAULT_CASE)
    ap.add_argument("--autotune", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-SGS form")
    ap.add_argument("--ensemble-branches", action="store_true",
                    help="ensemble: one CUDA-graph branch per member instead of the work-list launches")
    ap.add_argument("--no-extra", action="store_true",
                    help="headline case only (by default a one-GPU run of it also measures the ensemble and "
                         "the 1024x1024x256 domain)")
    args = ap.parse_args(argv)
    rank, world, local = dist_env()
    if world > 1:
        import datetime

        import torch.distributed as dist

        backend = "nccl" if args.impl == "ours" else "gloo"
        if backend == "nccl":
            import torch

            torch.cuda.set_device(local)
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
    try:
        if args.impl == "reference":
            line = run_reference(args, rank, world)
        elif args.case == ENSEMBLE_CASE:
            line = run_ensemble(args, rank, world, local)
        else:
            line = run_ours(args, rank, world, local)
            if line is not None and world == 1 and args.case == DEFAULT_CASE and not args.no_extra:
                try:
                    line["other_configs"] = other_configs(args, local)
                except Exception as exc:  # the headline line stands without them
                    line["other_configs"] = {"error": f"{type(exc).__name__}: {str(exc).splitlines()[0][:200]}"}
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
