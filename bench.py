#!/usr/bin/env python
"""Benchmark of the fused moment-representation LBM step on B200.

    python bench.py [--gpus N --steps K --warmup W] [--workload NAME] [--impl reference]

Default workload: D3Q27 lid-driven cavity, 256^3 nodes, Re = 1000,
u_lid = 0.05, with the function objects S, SMean, k and kMean updated every
step (FP32 storage, arithmetic and means, as the reference).  One step = one
time step of the whole cavity.  Prints one JSON line (rank 0).

* value       MLUPS of the device-timed step loop (CUDA events on the solver's
              stream, inputs resident in HBM; the moment buffers, 1.3 GB, are
              far larger than the 126 MB L2, so no flush is needed).
* e2e         the same metric through the C ABI with host buffers, one
              lbm_run_streamed call: upload of the state from pinned host
              memory, K steps (each step's 24-byte FP64 sums -- mass, kinetic
              energy, non-finite count -- copied back), download of the
              moments and function objects to pinned memory, the copies
              overlapping the steps -- all inside the timed region.  The
              same job as separate calls (lbm_write_fields, K x
              lbm_step_monitored, lbm_read_fields) is reported beside it.
* roofline    algorithmic bytes per node update (reference tiling: 134 B for
              D3Q27 + 4 + 24 + 48 + 8 B for k, S, SMean, kMean = 218 B) times
              the nodes per launch over the measured launch time, against the
              measured HBM copy bandwidth.
* other_workloads  plain D3Q27 / D3Q19 256^3, D3Q19 64^3, D3Q19 768^3 in FP32
              and FP16 storage and the 64-cavity batch, device-timed the same
              way in the same run, after the headline (--others '' skips them).
* cpu_baseline  the FP64 OpenMP CPU oracle (oracle/, a restatement of the
              reference's scheme; the reference has no CPU path) timed on this
              host on the same mesh for a bounded number of steps.

Multi-GPU: the cavity does not shard here ("replicas only"): every rank runs
its own cavity, no data-path collective; value = all ranks' node updates over
the slowest rank's time.

--impl reference runs the reference's own solver, built from its sources into
oracle/_ref (its only implementation is CUDA), on the same case, timing K steps
from its progress lines (printed every K steps, the first timed one at the
first multiple of K at or after W).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MLUPS and % HBM roofline (D3Q19/27 cavity); closure vs plain at equal error"

# B_alg: algorithmic bytes per node update at the reference tiling (8^3 blocks):
# moments 2*10*4 B + halo faces 2*0.75*QF*4 B (+ function-object traffic).
WORKLOADS = {
    "q27_256_fo": dict(lattice=27, n=(256, 256, 256), Re=1000.0, u=0.05, fo=("S", "SMean", "k", "kMean"),
                       mean_bits=32, b_alg=218,
                       desc="D3Q27 lid-driven cavity 256^3, Re=1000, u_lid=0.05, function objects S/SMean/k/kMean "
                            "every step (FP32 means)"),
    "q19_64": dict(lattice=19, n=(64, 64, 64), Re=100.0, u=0.05, fo=(), mean_bits=32, b_alg=110,
                   desc="D3Q19 lid-driven cavity 64^3, Re=100, u_lid=0.05"),
    "q19_256": dict(lattice=19, n=(256, 256, 256), Re=1000.0, u=0.05, fo=(), mean_bits=32, b_alg=110,
                    desc="D3Q19 lid-driven cavity 256^3, Re=1000, u_lid=0.05"),
    "q27_256": dict(lattice=27, n=(256, 256, 256), Re=1000.0, u=0.05, fo=(), mean_bits=32, b_alg=134,
                    desc="D3Q27 lid-driven cavity 256^3, Re=1000, u_lid=0.05"),
    "q19_512": dict(lattice=19, n=(512, 512, 512), Re=1000.0, u=0.05, fo=(), mean_bits=32, b_alg=110,
                    desc="D3Q19 lid-driven cavity 512^3, Re=1000, u_lid=0.05"),
    "q27_128_fo": dict(lattice=27, n=(128, 128, 128), Re=1000.0, u=0.05, fo=("S", "SMean", "k", "kMean"),
                       mean_bits=32, b_alg=218,
                       desc="D3Q27 lid-driven cavity 128^3, Re=1000, function objects S/SMean/k/kMean (profiling size)"),
    "q19_128": dict(lattice=19, n=(128, 128, 128), Re=1000.0, u=0.05, fo=(), mean_bits=32, b_alg=110,
                    desc="D3Q19 lid-driven cavity 128^3, Re=1000 (profiling size)"),
    "q19_768": dict(lattice=19, n=(768, 768, 768), Re=1000.0, u=0.05, fo=(), mean_bits=32, b_alg=110,
                    desc="D3Q19 lid-driven cavity 768^3, Re=1000, u_lid=0.05, FP32 moments"),
    "q19_768_f16": dict(lattice=19, n=(768, 768, 768), Re=1000.0, u=0.05, fo=(), mean_bits=32, b_alg=55,
                        storage="f16", desc="D3Q19 lid-driven cavity 768^3, Re=1000, u_lid=0.05, FP16 moment storage"),
    "q19_768_bf16": dict(lattice=19, n=(768, 768, 768), Re=1000.0, u=0.05, fo=(), mean_bits=32, b_alg=55,
                         storage="bf16", desc="D3Q19 lid-driven cavity 768^3, Re=1000, u_lid=0.05, BF16 moment storage"),
    "batch64_q19": dict(kind="batch", lattice=19, n_cav=64, seed=0, Re=None, u=0.05, fo=(), b_alg=110,
                        desc="64 D3Q19 cubic lid-driven cavities in one persistent launch per step (CUDA graph): "
                             "MT19937-64 seed 0 draws edges from {32,48,64,96,128} and Re from U[100,2000], "
                             "u_lid=0.05, FP32"),
    "closure_q27_128": dict(kind="closure", lattice=27, nc=128, u=0.05, tau=0.5077, fo=(), b_alg=134,
                            desc="learned closure: D3Q27 cavity 128^3 at tau 0.5077 (Re 2474) with the trained "
                                 "relaxation-time network, against plain 128^3 and plain 256^3 over the same "
                                 "physical time (10,000 coarse steps)"),
    "q27_256_fo64": dict(lattice=27, n=(256, 256, 256), Re=1000.0, u=0.05, fo=("S", "SMean", "k", "kMean"),
                         mean_bits=64, b_alg=274,
                         desc="D3Q27 lid-driven cavity 256^3, Re=1000, function objects with FP64 means"),
}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# --------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.25)

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        mhz, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        with open(self.path) as fh:
            for line in fh:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    mhz.append(float(parts[1]))
                    mx = float(parts[2])
                except ValueError:
                    continue
                for nm, val in zip(names, parts[5:9]):
                    if val.lower() == "active":
                        reasons.add(nm)
        os.unlink(self.path)
        if not mhz:
            return None
        return {"sm_mhz": statistics.median(mhz), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(mhz)}


def physical_gpu_index(local: int) -> int:
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [v for v in vis.split(",") if v.strip()]
        if local < len(ids) and ids[local].strip().isdigit():
            return int(ids[local])
    return local


def hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_per_node(workload: str):
    """DRAM bytes per node update of the step kernel from a committed ncu
    capture summary (profiles/traffic.json), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as fh:
            return float(json.load(fh)[workload]["dram_bytes_per_node"])
    except Exception:
        return None


# ----------------------------------------------------------- CPU oracle
def cpu_baseline(w, budget_s: float = 12.0):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    from pyoracle import Oracle

    from cudalbm_b200 import casefiles

    nx, ny, nz = w["n"]
    o = Oracle(w["lattice"], nx, ny, nz, w["Re"], w["u"])
    m = o.initial(casefiles.scaled_region_values(casefiles.lid_cavity_values(w["u"])))
    fo = o.new_function_objects(w["fo"])
    t0 = time.perf_counter()
    o.run(m, 1, 0, fo)
    one = time.perf_counter() - t0
    steps = max(1, min(5, int(budget_s / max(one, 1e-6)) - 1))
    t0 = time.perf_counter()
    o.run(m, steps, 1, fo)
    dt = time.perf_counter() - t0
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": round(nx * ny * nz * steps / dt / 1e6, 3), "unit": "MLUPS", "cores": cores, "kind": "port",
            "sample": f"FP64 OpenMP oracle, {w['desc']}, {steps} steps after 1 untimed"}


def link_ceiling(device: int):
    """Pinned host<->device copy rate of this box (GB/s): the best of three
    plain 1 GiB cudaMemcpyAsync each way, timed with CUDA events (torch is the
    plumbing here; the library is not involved)."""
    try:
        import torch

        n = 1 << 30
        dev = torch.device("cuda", device)
        torch.cuda.set_device(dev)
        h = torch.empty(n, dtype=torch.uint8, pin_memory=True)
        d = torch.empty(n, dtype=torch.uint8, device=dev)
        out = {}
        for key, fn in (("h2d", lambda: d.copy_(h, non_blocking=True)), ("d2h", lambda: h.copy_(d, non_blocking=True))):
            best = None
            for _ in range(3):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize(dev)
                e0.record()
                fn()
                e1.record()
                torch.cuda.synchronize(dev)
                ms = e0.elapsed_time(e1)
                best = ms if best is None else min(best, ms)
            out[key] = round(n / (best / 1e3) / 1e9, 2)
        # both directions at once (what an overlapped job sees): 1 GiB each way
        h2 = torch.empty(n, dtype=torch.uint8, pin_memory=True)
        d2 = torch.empty(n, dtype=torch.uint8, device=dev)
        s1, s2 = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
        best = None
        for _ in range(3):
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            with torch.cuda.stream(s1):
                d.copy_(h, non_blocking=True)
            with torch.cuda.stream(s2):
                h2.copy_(d2, non_blocking=True)
            torch.cuda.synchronize(dev)
            dt = time.perf_counter() - t0
            best = dt if best is None else min(best, dt)
        out["duplex_each_way"] = round(n / best / 1e9, 2)
        del h, d, h2, d2
        torch.cuda.empty_cache()
        return out
    except Exception as exc:  # reported, never silent
        log(f"link ceiling not measured: {exc!r}")
        return None


L2_BYTES = 126e6


def l2_note(buffer_bytes):
    """How the timed loop stands to the 126 MB L2 (no flush between steps)."""
    if buffer_bytes > L2_BYTES:
        return "inputs larger than L2 (moment buffers %.2f GB vs 126 MB L2); no flush" % (buffer_bytes / 1e9)
    return ("moment buffers %.3f GB fit in the 126 MB L2: the steps run L2-resident, no flush between them "
            "(the HBM fraction is not a bound at this size)" % (buffer_bytes / 1e9))


# ------------------------------------------------------------ our arm
def run_ours(args, w):
    import numpy as np

    from cudalbm_b200.replicas import Replicas

    group = Replicas("nccl")
    world, rank, local = group.world, group.rank, group.local
    barrier, max_over_ranks = group.barrier, group.max

    from cudalbm_b200 import _lib
    from cudalbm_b200.solver import NVARS, Cavity

    nx, ny, nz = w["n"]
    nodes = nx * ny * nz
    tile = (args.tile_x, args.tile_y, args.stages) if args.tile_x else None
    cav = Cavity(w["lattice"], nx, ny, nz, w["Re"], w["u"], function_objects=w["fo"], mean_bits=w["mean_bits"],
                 device=local, tile=tile, z_chunk=args.z_chunk, pop_buffers=args.pop_buffers,
                 storage=w.get("storage", "f32"))
    cav.init_regions()
    tuning = cav.autotune(args.tune_steps) if (not args.no_autotune and not args.tile_x) else None
    cav.step(args.warmup)
    cav.synchronize()

    # ---- device-timed loop (value)
    sampler = ClockSampler(physical_gpu_index(local))
    sampler.start()
    barrier()
    cav.synchronize()
    launches0 = cav.info()["kernel_launches"]
    cav.step(args.steps)
    cav.synchronize()
    barrier()
    info = cav.info()
    clocks = sampler.stop()
    ms = max_over_ranks(info["last_step_ms"])
    launches = info["kernel_launches"] - launches0
    ms_step = ms / args.steps
    value = world * nodes * args.steps / (ms / 1e3) / 1e6

    # ---- end to end through the C ABI with pinned host buffers (e2e)
    state = _lib.PinnedArray((10, nz, ny, nx), np.float32)  # host values are FP32 for every storage format
    cav.read("moments", out=state.array)
    outs = {fs: _lib.PinnedArray((NVARS[fs], nz, ny, nx), np.float64 if (w["mean_bits"] == 64 and "Mean" in fs)
                                 else np.float32) for fs in ("moments",) + tuple(w["fo"])}
    mon = _lib.PinnedArray((args.steps,), np.dtype(_lib.MONITOR_DTYPE))
    link = link_ceiling(local)
    # (a) the calls one after the other: upload, K monitored steps, download
    barrier()
    cav.synchronize()
    t0 = time.perf_counter()
    cav.write(state.array)
    t1 = time.perf_counter()
    for s in range(args.steps):
        cav.step_monitored(1, out=mon.array[s:s + 1])
    cav.synchronize()
    t2 = time.perf_counter()
    for fs, buf in outs.items():
        cav.read(fs, out=buf.array)
    t3 = time.perf_counter()
    barrier()
    seq_s = max_over_ranks(t3 - t0)
    h2d = 10 * nodes * 4
    d2h = sum(b.array.nbytes for b in outs.values())
    copy_gbs = {"h2d": round(h2d / (t1 - t0) / 1e9, 2), "d2h": round(d2h / (t3 - t2) / 1e9, 2)}
    red = {"mass": float(mon.array[-1]["mass"]), "nonfinite": int(mon.array["nonfinite"].max())}
    # (b) the same job as one lbm_run_streamed call: the upload, the steps
    # and the download overlap (z-slabs of each step shifted by the step
    # index).  One untimed call first (streams, events, staging).
    host_outs = {fs: b.array for fs, b in outs.items()}
    cav.run_streamed(state.array, min(args.steps, 4), host_outs, monitor=mon.array, slab=args.stream_slab,
                     z_chunk=args.stream_zc, lead=args.stream_lead)
    barrier()
    cav.synchronize()
    t4 = time.perf_counter()
    cav.run_streamed(state.array, args.steps, host_outs, monitor=mon.array, slab=args.stream_slab,
                     z_chunk=args.stream_zc, lead=args.stream_lead)
    t5 = time.perf_counter()
    barrier()
    e2e_s = max_over_ranks(t5 - t4)
    red = {"mass": float(mon.array[-1]["mass"]), "nonfinite": int(mon.array["nonfinite"].max())}
    e2e = world * nodes * args.steps / e2e_s / 1e6
    cav.close()
    group.close()

    if rank != 0:
        return None
    peak, peak_kind = hbm_peak()
    achieved = w["b_alg"] * nodes / (ms_step / 1e3) / 1e9
    tpn = traffic_per_node(args.workload)
    line = {
        "metric": METRIC,
        "value": round(value, 2),
        "unit": "MLUPS",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_step, 5),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": {"f32": "f32", "f16": "f16 storage, f32 arithmetic", "bf16": "bf16 storage, f32 arithmetic"}[
            w.get("storage", "f32")],
        "data": "synthetic: the lid-driven cavity initial state generated from the case's region values",
        "config": {"workload": w["desc"], "lattice": f"D3Q{w['lattice']}", "nx": nx, "ny": ny, "nz": nz,
                   "Re": w["Re"], "u_lid": w["u"], "function_objects": list(w["fo"]),
                   "mean_bits": w["mean_bits"], "parallelism": f"replicas x{world}",
                   "storage": w.get("storage", "f32"),
                   "l2": l2_note(2 * 10 * (2 if w.get("storage", "f32") != "f32" else 4) * nodes)},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": (round(tpn * nodes) if tpn else None),
                     "bytes_per_node_alg": w["b_alg"], "peak_kind": f"of {peak_kind}"},
        "e2e": {"value": round(e2e, 2), "unit": "MLUPS", "h2d_bytes_per_step": round(h2d / args.steps),
                "d2h_bytes_per_step": round(24 + d2h / args.steps),
                "what": ("one lbm_run_streamed call: pinned h2d of the state, K steps (each step's 24 B FP64 "
                         "mass/energy/non-finite sums), d2h of the moments and function objects, the copies "
                         "overlapping the steps"),
                "seconds": round(e2e_s, 5),
                "sequential": {"value": round(world * nodes * args.steps / seq_s / 1e6, 2),
                               "what": ("the same job as separate calls, one after the other: lbm_write_fields, "
                                        "K x lbm_step_monitored, lbm_read_fields of moments and function objects"),
                               "seconds": {"h2d": round(t1 - t0, 5), "steps": round(t2 - t1, 5),
                                           "d2h": round(t3 - t2, 5)},
                               "copy_gbs": copy_gbs},
                "link_gbs": link,
                "copy_frac_of_link": ({k: round(copy_gbs[k] / link[k], 3) for k in ("h2d", "d2h")}
                                      if link else None),
                "transfer_bound_mlups": (round(nodes * args.steps / (max(h2d / (link["h2d"] * 1e9),
                                                                         d2h / (link["d2h"] * 1e9))) / 1e6, 1)
                                         if link else None)},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "check": {"mass_last_step": red["mass"], "nonfinite_max": red["nonfinite"]},
        "kernel": {"tile": [info["tile_x"], info["tile_y"]], "z_chunk": info["z_chunk"], "stages": info["stages"],
                   "autotuned": tuning},
    }
    if world == 1 and args.others:
        line["other_workloads"] = other_workloads(args, local)
    if world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline(w)
        except Exception as exc:  # reported, never silent
            line["cpu_baseline"] = {"value": None, "error": repr(exc)}
    return line


OTHER_WORKLOADS = ("q27_256", "q19_256", "q19_64", "q19_768", "q19_768_f16", "batch64_q19")


def other_workloads(args, local):
    """The plain-method configurations beside the headline one, device-timed
    the same way (autotuned, W warm-up steps, K timed steps), so that their
    numbers come from the same run: D3Q27 and D3Q19 256^3 (the plain FP32
    roofline targets), D3Q19 64^3 (the small configuration), D3Q19 768^3 in
    FP32 and FP16 storage (the precision configuration) and the 64-cavity
    batch (one persistent launch per step).  They run after the headline
    measurement, so its clocks are not affected by theirs."""
    from cudalbm_b200 import casefiles
    from cudalbm_b200.solver import Batch, Cavity

    peak, peak_kind = hbm_peak()
    out = []
    for name in args.others.split(","):
        w = WORKLOADS[name]
        esz = 2 if w.get("storage", "f32") != "f32" else 4
        try:
            if w.get("kind") == "batch":
                specs = casefiles.random_cavities(w["n_cav"], seed=w["seed"], lattice=w["lattice"], u_lid=w["u"])
                nodes = sum(c["nx"] * c["ny"] * c["nz"] for c in specs)
                b = Batch(specs, device=local)
                b.init_regions()
                b.autotune(args.tune_steps)
                b.step(args.warmup)
                b.synchronize()
                b.step(args.steps)
                b.synchronize()
                info = b.info()
                b.close()
                kernel = {"tile": [info["tile_x"], info["tile_y"]], "persistent": info["persistent"]}
            else:
                nx, ny, nz = w["n"]
                nodes = nx * ny * nz
                cav = Cavity(w["lattice"], nx, ny, nz, w["Re"], w["u"], function_objects=w["fo"],
                             mean_bits=w["mean_bits"], device=local, storage=w.get("storage", "f32"))
                cav.init_regions()
                cav.autotune(args.tune_steps)
                cav.step(args.warmup)
                cav.synchronize()
                cav.step(args.steps)
                cav.synchronize()
                info = cav.info()
                cav.close()
                kernel = {"tile": [info["tile_x"], info["tile_y"]], "z_chunk": info["z_chunk"],
                          "stages": info["stages"]}
        except Exception as exc:  # reported, never silent
            out.append({"workload": w["desc"], "error": repr(exc)})
            continue
        ms_step = info["last_step_ms"] / args.steps
        achieved = w["b_alg"] * nodes / (ms_step / 1e3) / 1e9
        out.append({"workload": w["desc"], "value": round(nodes / (ms_step / 1e3) / 1e6, 2), "unit": "MLUPS",
                    "ms_per_step": round(ms_step, 5), "roofline_frac": round(achieved / peak, 4),
                    "bytes_per_node_alg": w["b_alg"], "peak_kind": f"of {peak_kind}",
                    "physical_frac": round(20 * esz * nodes / (ms_step / 1e3) / 1e9 / peak, 4),
                    "kernel": kernel})
    return out


# ------------------------------------------------------ batched arm
def run_batch(args, w):
    """Aggregate MLUPS of many cavities advanced by one persistent launch per
    step, beside the same cavities stepped by one plain launch each, one after
    another on the same stream (the single-cavity path, each size class with
    its own autotuned kernel)."""
    import numpy as np

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        return {"impl": "ours", "unavailable": "the batched workload is measured on one GPU"} if rank == 0 else None

    from cudalbm_b200 import _lib, casefiles
    from cudalbm_b200.solver import Batch

    specs = casefiles.random_cavities(w["n_cav"], seed=w["seed"], lattice=w["lattice"], u_lid=w["u"])
    nodes = sum(c["nx"] * c["ny"] * c["nz"] for c in specs)
    b = Batch(specs, device=local)
    b.init_regions()
    tuning = None if args.no_autotune else b.autotune(args.tune_steps)
    b.step(args.warmup)
    b.synchronize()

    # ---- device-timed batched loop (value)
    sampler = ClockSampler(physical_gpu_index(local))
    sampler.start()
    launches0 = b.info()["kernel_launches"]
    b.step(args.steps)
    b.synchronize()
    info = b.info()
    clocks = sampler.stop()
    ms = info["last_step_ms"]
    ms_step = ms / args.steps
    value = nodes * args.steps / (ms / 1e3) / 1e6
    launches = info["kernel_launches"] - launches0

    # ---- the same cavities, one plain launch each per step (wall clock)
    for c in b.cavities:
        c.autotune(args.tune_steps)
    seq_steps = max(3, min(args.steps, 200))
    for c in b.cavities:
        c.step(1)
    b.synchronize()
    t0 = time.perf_counter()
    for _ in range(seq_steps):
        for c in b.cavities:
            c.step(1)
    b.synchronize()
    seq = nodes * seq_steps / (time.perf_counter() - t0) / 1e6
    t0 = time.perf_counter()
    b.step(seq_steps)
    b.synchronize()
    batch_wall = nodes * seq_steps / (time.perf_counter() - t0) / 1e6

    # ---- end to end through the C ABI with pinned host buffers
    states = [_lib.PinnedArray((10, c.shape[0], c.shape[1], c.shape[2]), np.float32) for c in b.cavities]
    for c, st in zip(b.cavities, states):
        c.read("moments", out=st.array)
    t0 = time.perf_counter()
    for c, st in zip(b.cavities, states):
        c.write(st.array)
    b.step(args.steps)
    for c, st in zip(b.cavities, states):
        c.read("moments", out=st.array)
    e2e_s = time.perf_counter() - t0
    e2e = nodes * args.steps / e2e_s / 1e6
    state_bytes = sum(st.array.nbytes for st in states)
    bad = sum(int(c.reduce()["nonfinite"]) for c in b.cavities)
    b.close()

    peak, peak_kind = hbm_peak()
    achieved = w["b_alg"] * nodes / (ms_step / 1e3) / 1e9
    edges = {}
    for c in specs:
        edges[c["nx"]] = edges.get(c["nx"], 0) + 1
    line = {
        "metric": METRIC,
        "value": round(value, 2),
        "unit": "MLUPS",
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_step, 5),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic: 64 lid-driven cavity initial states (seeded sizes and Reynolds numbers)",
        "config": {"workload": w["desc"], "lattice": f"D3Q{w['lattice']}", "cavities": len(specs), "nodes": nodes,
                   "edges": {str(k): v for k, v in sorted(edges.items())}, "parallelism": "1 GPU",
                   "l2": l2_note(80 * nodes)},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": None, "bytes_per_node_alg": w["b_alg"],
                     "peak_kind": f"of {peak_kind}"},
        "e2e": {"value": round(e2e, 2), "unit": "MLUPS", "h2d_bytes_per_step": round(state_bytes / args.steps),
                "d2h_bytes_per_step": round(state_bytes / args.steps),
                "what": "lbm_write_fields of every cavity (pinned h2d) + lbm_batch_step(K) + lbm_read_fields of "
                        "every cavity's moments"},
        "sequential": {"value": round(seq, 2), "unit": "MLUPS", "steps": seq_steps,
                       "what": "each step = 64 plain launches (one per cavity, autotuned per size class), one after "
                               "another on one stream; wall clock",
                       "batched_same_clock": round(batch_wall, 2),
                       "speedup": round(batch_wall / seq, 3)},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "check": {"nonfinite": bad},
        "kernel": {"tile": [info["tile_x"], info["tile_y"]], "stages": info["stages"],
                   "pop_buffers": info["pop_buffers"], "grid": info["grid"], "items": info["items"],
                   "graph_launches_timed": args.steps // 2, "autotuned": tuning},
    }
    if not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline(dict(lattice=19, n=(64, 64, 64), Re=specs[0]["Re"], u=w["u"], fo=(),
                                                     desc="one 64^3 D3Q19 cavity of the batch"))
        except Exception as exc:
            line["cpu_baseline"] = {"value": None, "error": repr(exc)}
    return line


# ------------------------------------------------------ closure arm
def run_closure(args, w):
    """The closure half of the metric: train the network (cudalbm_b200/
    closure_study.py), then time the learned coarse run and report its error
    and wall time beside the plain coarse and the plain fine (2x) runs.  value
    = the learned coarse run's device-timed MLUPS with the network evaluated
    on the tensor cores every step."""
    rank = int(os.environ.get("RANK", "0"))
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        return {"impl": "ours", "unavailable": "the closure study runs on one GPU"} if rank == 0 else None
    from cudalbm_b200.closure_study import run_study
    from cudalbm_b200.solver import Cavity

    study = run_study(nc=w["nc"], tau_coarse=w["tau"], log=lambda m: log(m))
    nc = w["nc"]
    Re = study["config"]["Re"]
    # device-timed learned steps (the study's network is not returned: retrain-free timing with a
    # constant-shape network gives the same instruction stream)
    from cudalbm_b200 import _lib

    net = _lib.MLP()
    net.in_lo[:] = [-1e30] * 16
    net.in_hi[:] = [1e30] * 16
    net.in_scale[:] = [1.0] * 16
    net.dtau_lo, net.dtau_hi = study["config"]["dtau_range"]
    with Cavity(w["lattice"], nc, nc, nc, Re, w["u"]) as c:
        c.init_regions()
        c.set_closure(net)
        c.step(args.warmup)
        c.synchronize()
        sampler = ClockSampler(physical_gpu_index(int(os.environ.get("LOCAL_RANK", "0"))))
        sampler.start()
        c.step(args.steps)
        c.synchronize()
        ms = c.info()["last_step_ms"]
        clocks = sampler.stop()
        launches = args.steps * 2
    nodes = nc ** 3
    value = nodes * args.steps / (ms / 1e3) / 1e6
    T = study["config"]["coarse_steps"]
    peak, peak_kind = hbm_peak()
    achieved = w["b_alg"] * nodes / (ms / args.steps / 1e3) / 1e9
    return {
        "metric": METRIC, "value": round(value, 2), "unit": "MLUPS", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 moments; f16 network weights/activations, f32 accumulate",
        "data": "synthetic: lid-driven cavity; training runs with U(-1e-3,1e-3) velocity perturbations, seeds 0-7",
        "config": {"workload": w["desc"], "lattice": f"D3Q{w['lattice']}", "nx": nc, "ny": nc, "nz": nc, "Re": Re,
                   "parallelism": "1 GPU", "l2": "moments 0.17 GB: close to L2; MLUPS of a small mesh"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": None, "bytes_per_node_alg": w["b_alg"],
                     "peak_kind": f"of {peak_kind}"},
        "e2e": {"value": round(nodes * study["learned"]["steps"] / study["learned"]["wall"] / 1e6, 2), "unit": "MLUPS",
                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": round(40 * nodes * 2 / study["learned"]["steps"]),
                "what": "the study's learned run through the public API, wall clock, with two state read-backs"},
        "closure": {"error_plain": study["plain"][T], "error_learned": study["learned"][T],
                    "wall_s": {"fine_plain": study["fine_wall_s"], "coarse_plain": study["plain"]["wall"],
                               "coarse_learned": study["learned"]["wall"]},
                    "speedup_learned_vs_fine": study["speedup_learned_vs_fine"], "training": study["training"]},
        "gpu_launches": launches, "clocks": clocks,
    }


# ------------------------------------------------------- reference arm
def reference_step_time(exe, spec, W, K, local):
    """Seconds per step of the reference executable on one case, from two of
    its 'Time:' progress lines K steps apart, the first at the first multiple
    of K at or after W (the case prints every K steps, so no per-step output
    is timed); (dt, clocks, error)."""
    from cudalbm_b200 import casefiles

    with tempfile.TemporaryDirectory() as case:
        casefiles.write_case(case, spec)
        sampler = ClockSampler(physical_gpu_index(local))
        proc = subprocess.Popen([exe, "-GPU", str(local)], cwd=case, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                                text=True, bufsize=1)
        stamps = {}
        tail = []
        clocks = None
        starter = None
        for line in proc.stdout:
            now = time.perf_counter()
            tail = (tail + [line])[-20:]
            if line.startswith("Time: "):
                t = int(line.split()[1])
                stamps[t] = now
                if t == W:
                    # started aside: reading (and stamping) the step lines never waits on the sampler
                    starter = threading.Thread(target=sampler.start)
                    starter.start()
                if t == W + K:
                    starter.join()
                    clocks = sampler.stop()
        rc = proc.wait()
        if starter is not None and clocks is None:
            starter.join()
            sampler.stop()
    if rc != 0 or W not in stamps or W + K not in stamps:
        return None, None, f"reference exited {rc}: {''.join(tail)[-300:]!r}"
    return (stamps[W + K] - stamps[W]) / K, clocks, None


def reference_case(spec_kw, W, K):
    """Case settings for reference_step_time: progress lines every K steps,
    timing from step W0 = the first multiple of K at or after W to W0 + K;
    returns (spec keyword arguments, W0)."""
    W0 = -(-W // K) * K
    return dict(spec_kw, n_steps=W0 + K + 1, save_interval=W0 + K + 10, info_interval=K), W0


def run_reference(args, w):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    from cudalbm_b200 import casefiles

    exe = os.path.join(ROOT, "oracle", "_ref", f"momentBasedD3Q{w['lattice']}")
    if not os.path.exists(exe):
        return {"impl": "reference", "unavailable": f"{exe} not built (make -f oracle/Makefile.ref needs the "
                                                    "reference sources)"}
    W, K = args.warmup, args.steps
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if w.get("kind") == "batch":
        # the reference runs one cavity per process: time each size class once
        # and charge every cavity of the batch its class's step time
        cavs = casefiles.random_cavities(w["n_cav"], seed=w["seed"], lattice=w["lattice"])
        per_edge, clocks = {}, None
        for e in sorted({c["nx"] for c in cavs}):
            c0 = next(c for c in cavs if c["nx"] == e)
            kw, W0 = reference_case(dict(nx=e, ny=e, nz=e, Re=c0["Re"], u_inf=w["u"]), W, K)
            dt, clk, err = reference_step_time(exe, casefiles.CaseSpec(**kw), W0, K, local)
            if err:
                return {"impl": "reference", "unavailable": err}
            per_edge[e] = dt
            clocks = clk or clocks
        nodes = sum(c["nx"] ** 3 for c in cavs)
        dt = sum(per_edge[c["nx"]] for c in cavs)
        cfg = {"workload": w["desc"], "lattice": f"D3Q{w['lattice']}", "cavities": len(cavs), "nodes": nodes,
               "parallelism": "1 GPU", "seconds_per_step_by_edge": {str(k): v for k, v in per_edge.items()}}
        sample = ("the reference's own executable run once per size class (one cavity per process, as it "
                  f"supports), {K} steps after {W} each, per-step times summed over the 64 cavities")
    else:
        if w.get("kind") == "closure":
            # the reference has no closure: its plain solver on the same coarse case
            nx = ny = nz = w["nc"]
            w = dict(w, n=(nx, ny, nz), Re=w["u"] * (nx - 1) / ((w["tau"] - 0.5) / 3.0))
        nx, ny, nz = w["n"]
        nodes = nx * ny * nz
        kw, W0 = reference_case(dict(nx=nx, ny=ny, nz=nz, Re=w["Re"], u_inf=w["u"], function_objects=w["fo"]), W, K)
        dt, clocks, err = reference_step_time(exe, casefiles.CaseSpec(**kw), W0, K, local)
        if err:
            return {"impl": "reference", "unavailable": err}
        cfg = {"workload": w["desc"], "lattice": f"D3Q{w['lattice']}", "nx": nx, "ny": ny, "nz": nz,
               "Re": w["Re"], "u_lid": w["u"], "function_objects": list(w["fo"]), "parallelism": "1 GPU"}
        sample = (f"the reference's own executable (oracle/_ref/momentBasedD3Q{w['lattice']}, built from its "
                  f"sources for sm_100a) on the B200 -- its only implementation is CUDA; {K} steps after "
                  f"{-(-W // K) * K} (the first multiple of K at or after W={W}), timed by two of its 'Time:' progress "
                  "lines, printed every K steps (wall clock; the reference synchronises the device every step)")
    value = nodes / dt / 1e6
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": round(value, 2),
        "unit": "MLUPS",
        "n_gpus": 1,
        "steps": K,
        "warmup": W,
        "ms_per_step": round(dt * 1e3, 5),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic: the same lid-driven cavity case directories",
        "config": cfg,
        "cpu_baseline": {"value": round(value, 2), "unit": "MLUPS", "cores": 1, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": round(value, 2), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "clocks": clocks,
    }


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=50)
    ap.add_argument("--workload", default="q27_256_fo", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tile-x", type=int, default=0, help="kernel tiling override (default: autotuned)")
    ap.add_argument("--tile-y", type=int, default=8)
    ap.add_argument("--stages", type=int, default=0)
    ap.add_argument("--z-chunk", type=int, default=0)
    ap.add_argument("--pop-buffers", type=int, default=0)
    ap.add_argument("--no-autotune", action="store_true", help="keep the default kernel variant")
    ap.add_argument("--tune-steps", type=int, default=10)
    ap.add_argument("--others", default=",".join(OTHER_WORKLOADS),
                    help="plain workloads also timed (device) in the default run, comma-separated; '' for none")
    ap.add_argument("--stream-slab", type=int, default=0, help="lbm_run_streamed slab height (0: default)")
    ap.add_argument("--stream-zc", type=int, default=0, help="lbm_run_streamed z-chunk (0: default)")
    ap.add_argument("--stream-lead", type=int, default=0, help="lbm_run_streamed first-slab lead (0: default)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    w = WORKLOADS[args.workload]
    if args.impl == "reference":
        line = run_reference(args, w)
    elif w.get("kind") == "batch":
        line = run_batch(args, w)
    elif w.get("kind") == "closure":
        line = run_closure(args, w)
    else:
        line = run_ours(args, w)
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
