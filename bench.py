"""Benchmark: D3Q19 BGK fused collide-and-stream on a periodic 256^3 Taylor-Green vortex.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

One step = one fused collide + periodic-shift stream over the whole 256^3 lattice (FP32
storage, nu = 0.01, u0 = 0.05), the bandwidth-roofline configuration of the reference's
benchmark set.  `value` is MLUPS with the populations resident in HBM; `e2e` is the same
metric through the C ABI with host buffers (upload of the initial populations from pinned
memory, every step's lattice statistics read back, download of the final populations).  The
FP16/BF16 deviation-storage and FP64 forms are timed beside it under "forms".  With N GPUs
every rank steps its own lattice (replicas; the path needs no collective) and `value`
aggregates over ranks with the max-over-ranks time.

--impl reference times the reference's own CPU implementation (OpenMP + SIMD build of
OpenLB, oracle/_ref) on this host's cores on the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "MLUPS (D3Q19 256^3 fused collide-and-stream)"
NU = 0.01
U0 = 0.05
OMEGA = 1.0 / (3.0 * NU + 0.5)
BYTES_PER_LUP = {"f64": 2 * 19 * 8, "f32": 2 * 19 * 4, "f16dev": 2 * 19 * 2, "bf16dev": 2 * 19 * 2}


def hbm_peak() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def profile_traffic() -> float | None:
    """dram read+write bytes per launch of the step kernel from the committed ncu summary."""
    p = ROOT / "profiles" / "k_collide_stream_d3q19_f32_256.md"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.strip().startswith("traffic_bytes_per_launch_256:"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


# ---------------------------------------------------------------------------------------------
# clocks sampler (nvidia-smi during the timed region)
class Clocks:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "10"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except FileNotFoundError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


# ---------------------------------------------------------------------------------------------
def reference_binary() -> Path | None:
    flags = ""
    try:
        flags = Path("/proc/cpuinfo").read_text()
    except OSError:
        pass
    isa = "avx512" if " avx512f" in flags and " avx512bw" in flags else "avx2"
    exe = ROOT / "oracle" / "_ref" / f"lbref_d3q19_f32_omp_{isa}"
    return exe if exe.exists() else None


def time_reference(n: int, warmup: int, steps: int, threads: int) -> dict:
    exe = reference_binary()
    if exe is None:
        raise FileNotFoundError("reference CPU build missing (make -C oracle ref)")
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="close", OMP_PLACES="cores")
    cmd = [str(exe), "periodic", "--n", str(n), str(n), str(n), "--dyn", "bgk", "--omega", repr(OMEGA),
           "--init", "tgv", "--u0", repr(U0), "--time", str(warmup), str(steps)]
    with __import__("tempfile").TemporaryDirectory() as tmp:
        out = subprocess.run(cmd, env=env, cwd=tmp, capture_output=True, text=True, timeout=900, check=True).stdout
    line = [l for l in out.splitlines() if l.startswith("{")][-1]
    r = json.loads(line)
    r["binary"] = exe.name
    return r


def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# ---------------------------------------------------------------------------------------------
def tgv_fields(n: int):
    x = 2 * np.pi * np.arange(n) / n
    sx, cx = np.sin(x), np.cos(x)
    ux = U0 * sx[:, None, None] * cx[None, :, None] * cx[None, None, :]
    uy = -U0 * cx[:, None, None] * sx[None, :, None] * cx[None, None, :]
    u = np.stack([ux.reshape(-1), uy.reshape(-1), np.zeros(n ** 3)])
    return np.ones(n ** 3), u


STEP_KERNEL = {0: "k_collide_stream_tiled", 1: "k_collide_stream", 2: "k_collide_stream_groups",
               3: "k_collide_stream_bulk", 4: "k_collide_stream_ws", 5: "k_collide_stream_groups"}


def current_config(tuning: list[dict]) -> dict:
    """The launch shape in use: the autotuner's pick (fastest timed candidate), else the default."""
    timed = [t for t in tuning if t["ms_per_step"] > 0]
    if not timed:
        return {"variant": 2, "block_x": None, "block_y": None, "cells_per_thread": 1, "source": "default"}
    best = min(timed, key=lambda t: t["ms_per_step"])
    return {k: best[k] for k in ("variant", "block_x", "block_y", "cells_per_thread")} | {"source": "autotune"}


def launch_config(cfg: dict, tuning: list[dict]) -> dict:
    out = dict(cfg)
    out["candidates"] = len(tuning)
    out["tuned_ms_per_step"] = {f"v{t['variant']}/{t['block_x']}x{t['block_y']}/k{t['cells_per_thread']}":
                                round(t["ms_per_step"], 4) for t in tuning}
    return out


def rank_max(dist, v: float, device: str = "cpu") -> float:
    """Max of a per-rank time over all ranks (every rank calls it; the replicas' job time is
    the slowest rank's)."""
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_mlups(world: int, cells: int, steps: int, max_ms: float) -> float:
    """Whole-job throughput of N replicas: every rank updates `cells` cells `steps` times; the
    job takes the slowest rank's time."""
    return world * cells * steps / (max_ms * 1e-3) / 1e6


def run_b200(args, rank: int, world: int, device: int, dist) -> dict | None:
    import torch

    from openlb_b200 import lbx

    torch.cuda.set_device(device)
    stream = torch.cuda.Stream(device=device)
    n = args.size
    cells = n ** 3
    rho, u = tgv_fields(n)

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(v: float) -> float:
        return rank_max(dist, v, f"cuda:{device}")

    def timed_steps(lat, k: int) -> float:
        """ms for k fused steps, device-timed on the launch stream, max over ranks."""
        barrier()
        torch.cuda.synchronize(device)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        lat.collide_and_stream(k, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize(device)
        barrier()
        return max_over_ranks(e0.elapsed_time(e1))

    # ---- headline: FP32 storage, populations resident -----------------------------------------
    lat = lbx.BlockLattice(19, (n, n, n), (1, 1, 1), args.storage, device=device)
    lat.define_dynamics("bgk", omega=OMEGA)
    lat.ini_equilibrium(rho, u, stream=stream)
    lat.collide_and_stream(args.warmup, stream=stream)
    tuning = lat.autotune(steps=30, stream=stream) if not (args.no_autotune or args.launch_config) else []
    if args.launch_config:
        lat.set_launch_config(*args.launch_config)
        tuning = [{"variant": args.launch_config[0], "block_x": args.launch_config[1],
                   "block_y": args.launch_config[2], "cells_per_thread": args.launch_config[3],
                   "ms_per_step": 1.0}]
    torch.cuda.synchronize(device)
    clocks = Clocks(device)
    clocks.start()
    ms = timed_steps(lat, args.steps)
    # the same steps again with events around each kernel: the step kernel's own duration
    lat.set_kernel_timing(True)
    timed_steps(lat, args.steps)
    kt = lat.kernel_timing()
    lat.set_kernel_timing(False)
    lat_cfg = current_config(tuning)
    if args.launch_config:
        lat_cfg["source"] = "fixed (--launch-config)"
    per_step_ms = ms / args.steps
    mlups = job_mlups(world, cells, args.steps, ms)
    coll_ms, coll_n = kt["collision"]
    halo_ms, halo_n = kt["periodic_overlap"]
    launch_s = coll_ms / max(coll_n, 1) * 1e-3
    bytes_launch = cells * BYTES_PER_LUP[args.storage]
    peak, peak_kind = hbm_peak()
    achieved_gbs = bytes_launch / launch_s / 1e9
    lat.collide_and_stream(1, statistics=True, stream=stream)
    stats = lat.get_statistics(stream=stream)

    # ---- e2e through the C ABI with host buffers -----------------------------------------------
    f_host = torch.empty((19, cells), dtype=torch.float32 if args.storage != "f64" else torch.float64,
                         pin_memory=True)
    f_np = f_host.numpy()
    lat.get_populations(out=f_np, stream=stream)
    barrier()
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    lat.set_populations(f_np, stream=stream)
    for _ in range(args.steps):
        lat.collide_and_stream(1, statistics=True, stream=stream)
        lat.get_statistics(stream=stream)
    lat.get_populations(out=f_np, stream=stream)
    torch.cuda.synchronize(device)
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    barrier()
    # the sampler ran through the three timed sections (resident steps, per-kernel timing, e2e)
    clk = clocks.stop()
    e2e_mlups = job_mlups(world, cells, args.steps, e2e_s * 1e3)
    pop_bytes = f_np.nbytes
    lat.close()

    # ---- other storage forms (shorter runs) ------------------------------------------------------
    forms = {}
    fields = {}
    if not args.no_forms:
        for form in ("f16dev", "bf16dev", "f32", "f64"):
            k = max(10, args.steps // 4)
            fl = lbx.BlockLattice(19, (n, n, n), (1, 1, 1), form, device=device)
            fl.define_dynamics("bgk", omega=OMEGA)
            fl.ini_equilibrium(rho, u, stream=stream)
            fl.collide_and_stream(args.warmup, stream=stream)
            f_tuning = fl.autotune(steps=30, stream=stream) if not args.no_autotune else []
            fms = timed_steps(fl, k)
            fl.set_kernel_timing(True)
            timed_steps(fl, k)
            fk_ms, fk_n = fl.kernel_timing()["collision"]
            f_mlups = job_mlups(world, cells, k, fms)
            f_gbs = cells * BYTES_PER_LUP[form] / (fk_ms / max(fk_n, 1) * 1e-3) / 1e9
            forms[form] = {"mlups": round(f_mlups, 1), "hbm_gbs": round(f_gbs, 1),
                           "hbm_frac": round(f_gbs / peak, 4), "vs_f32_mlups": round(f_mlups / mlups, 3),
                           "steps": k, "launch_config": current_config(f_tuning)}
            f_rho, f_u = fl.compute_moments(stream=stream)
            fields[form] = (f_rho.astype(np.float64), f_u.astype(np.float32 if form != "f64" else np.float64))
            del f_rho, f_u
            fl.close()
        # accuracy of every storage form against the FP64 run after the same steps from the same
        # initial state (the FP64 kernel reproduces the reference's FP64 arithmetic)
        rho64, u64 = fields["f64"]
        for form in ("f16dev", "bf16dev", "f32"):
            r, uu = fields[form]
            du = uu.astype(np.float64) - u64
            forms[form]["error_vs_f64"] = {
                "u_l2_rel": float(np.sqrt((du ** 2).sum() / (u64 ** 2).sum())),
                "u_linf_rel": float(np.abs(du).max() / np.abs(u64).max()),
                "rho_linf": float(np.abs(r - rho64).max()),
                "after_steps": int(args.warmup + 2 * max(10, args.steps // 4))}
        del fields
        # against the FP32 form's own run of the same length (vs_f32_mlups: against the headline)
        for form in forms:
            forms[form]["vs_f32_form_mlups"] = round(forms[form]["mlups"] / forms["f32"]["mlups"], 3)

    ensemble = None if args.ensemble_requests <= 0 else run_ensemble(args, device, stream)

    if rank != 0:
        return None
    # the committed capture covers the FP32 256^3 step kernel; other workloads have no figure
    traffic = profile_traffic() if (n == 256 and args.storage == "f32") else None
    line = {
        "metric": METRIC, "value": round(mlups, 1), "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(per_step_ms, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32" if args.storage != "f64" else "f64",
        "data": "synthetic (Taylor-Green vortex initial state, seeded-free analytic field)",
        "config": {"workload": f"D3Q19 BGK periodic {n}^3 Taylor-Green u0={U0} nu={NU}, {args.storage} storage",
                   "cells": cells, "storage": args.storage, "parallelism": "replicas" if world > 1 else "single",
                   "l2": f"population arrays {bytes_launch / 2 / 1e9:.2f} GB > 126 MB L2; no flush needed"},
        "roofline": {"bound": "hbm", "achieved": round(achieved_gbs, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved_gbs / peak, 4), "peak_kind": peak_kind,
                     "traffic": traffic, "algorithmic_bytes_per_launch": bytes_launch},
        "e2e": {"value": round(e2e_mlups, 1), "unit": "MLUPS", "h2d_bytes_per_step": int(pop_bytes / args.steps),
                "d2h_bytes_per_step": int(pop_bytes / args.steps + 32)},
        "gpu_launches": coll_n + halo_n,
        "launch_config": launch_config(lat_cfg, tuning),
        "kernels": {k: v for k, v in {
            STEP_KERNEL[lat_cfg["variant"]]: {"avg_ms": round(coll_ms / max(coll_n, 1), 5), "launches": coll_n,
                                        "share": round(coll_ms / max(coll_ms + halo_ms, 1e-12), 4)},
            "k_periodic_halo": {"avg_ms": round(halo_ms / max(halo_n, 1), 5), "launches": halo_n,
                                "share": round(halo_ms / max(coll_ms + halo_ms, 1e-12), 4)}}.items()
            if v["launches"] > 0},
        "clocks": clk,
        "statistics": stats,
        "forms": forms,
    }
    if ensemble is not None:
        line["ensemble"] = ensemble
    return line


def run_ensemble(args, device: int, stream) -> dict:
    """Serving form: a bounded sample of the lid-driven cavity parameter sweep (D3Q19 BGK, FP32,
    edges {32..192}, Re log-uniform [10, 1000], lid 0.05, Poisson arrivals at 200/s, residual
    tolerance 1e-6 with the step count capped) served by the continuous-batching ensemble server,
    then the same requests solved one after another on the single-lattice path."""
    import torch

    from openlb_b200 import lbx, serving

    reqs = serving.sample_requests(args.ensemble_requests, seed=2024, max_steps=args.ensemble_max_steps)
    check = 100
    # the slab holds about 40 % of the sample's total footprint (at least the largest request),
    # so requests wait for memory and are admitted as earlier ones retire
    foot = [lbx.Ensemble.footprint_of(19, "f32", r.engine_request()) for r in reqs]
    slab = max(int(1.05 * max(foot)), int(0.4 * sum(foot)))
    slab = (slab + (1 << 20) - 1) >> 20 << 20
    with lbx.Ensemble(19, "f32", slab_bytes=max(slab, 1 << 30), max_lattices=256, device=device) as ens:
        ens.set_config(threads=256, blocks_per_sm=0, check_interval=check)
        # tune the persistent kernel once on one cavity of every edge length, then empty the slab
        probe = [ens.admit(serving.CavityRequest(i, e, 100.0).engine_request())
                 for i, e in enumerate((32, 48, 64, 96, 128, 192))]
        tuning = ens.autotune(steps=10, stream=stream)
        for slot in probe:
            ens.retire(slot)
        timed = [t for t in tuning if t["ms_per_step"] > 0]
        pick = min(timed, key=lambda t: t["ms_per_step"]) if timed else None
        server = serving.EnsembleServer(ens, chunk=500, min_chunk=check, stream=stream)
        serving_warm = serving.sample_requests(4, seed=1, edges=(16,), max_steps=1000)
        server.serve(serving_warm, realtime=False)  # graph capture and first-launch costs
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        recs = server.serve(reqs)
        torch.cuda.synchronize(device)
        wall = time.perf_counter() - t0
        loop_stats = server.last_stats
    served = serving.summarise(recs, wall)
    served["slab_bytes"] = int(max(slab, 1 << 30))
    served["sample_footprint_bytes"] = int(sum(foot))
    served["runs"] = {k: loop_stats[k] for k in ("runs", "short_runs", "long_runs", "steps")}
    served["loop"] = "native (lbx_server_*): first-fit admission by footprint, adaptive chunk 100/500 steps"
    t0 = time.perf_counter()
    seq = serving.solve_sequential(reqs, check_interval=check, device=device)
    torch.cuda.synchronize(device)
    seq_wall = time.perf_counter() - t0
    sequential = serving.summarise(seq, seq_wall)
    return {"workload": f"{len(reqs)} D3Q19 BGK lid-driven cavity requests, edge ~ U{{32,48,64,96,128,192}}, "
                        f"Re ~ logU[10,1000], lid 0.05, Poisson 200/s (seed 2024), stop at L2 velocity "
                        f"residual < 1e-6 (delta {check} steps) or {args.ensemble_max_steps} steps; f32 storage",
            "sample": f"{len(reqs)} requests with the step cap lowered from 50000 to {args.ensemble_max_steps} "
                      f"so the run ends in seconds; slab = 40 % of their total footprint",
            "sequential_setup": "one lattice created per request; host cell map and link list derived once per "
                                "cavity size and reused",
            "launch_config": None if pick is None else {"launch_mode": ("persistent" if pick["variant"] == 0
                                                                        else "graph of step launches"),
                                                        "threads": pick["threads"],
                                                        "blocks_per_sm": pick["blocks_per_sm"],
                                                        "candidates": len(tuning), "source": "autotune"},
            "server": served, "sequential": sequential,
            "speedup_vs_sequential": round(sequential["wall_s"] / served["wall_s"], 3)}


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--storage", default="f32", choices=["f32", "f64", "f16dev", "bf16dev"])
    ap.add_argument("--no-forms", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--launch-config", type=int, nargs=4, metavar=("VARIANT", "BX", "BY", "K"),
                    help="fixed launch shape of the headline lattice instead of the autotuner's")
    ap.add_argument("--ensemble-requests", type=int, default=32)
    ap.add_argument("--ensemble-max-steps", type=int, default=2000)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        threads = os.cpu_count() or 1
        k, w = args.steps, args.warmup
        r = time_reference(args.size, w, k, threads)
        line = {"impl": "reference", "metric": METRIC, "value": round(r["mlups"], 2), "unit": "MLUPS",
                "n_gpus": args.gpus, "steps": k, "warmup": w, "ms_per_step": round(1e3 * r["seconds"] / k, 3),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (Taylor-Green vortex initial state)",
                "config": {"workload": f"D3Q19 BGK periodic {args.size}^3 Taylor-Green u0={U0} nu={NU}, f32 storage",
                           "cells": args.size ** 3, "storage": "f32", "parallelism": "host cores"},
                "cpu_baseline": {"value": round(r["mlups"], 2), "unit": "MLUPS", "cores": r["threads"],
                                 "kind": "reference",
                                 "sample": f"{args.size}^3 lattice, {w} warm-up + {k} timed steps of OpenLB "
                                           f"CPU_SIMD+OpenMP ({r['binary']}) on {cpu_model()}"},
                "e2e": {"value": round(r["mlups"], 2), "unit": "MLUPS", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist

        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                 device_id=torch.device(f"cuda:{local}"))
        dist = tdist
    line = run_b200(args, rank, world, local, dist)
    if line is not None and world == 1 and not args.no_cpu_baseline:
        try:
            threads = os.cpu_count() or 1
            # the arm's step counts, bounded to about half a minute of CPU work
            k, w = min(args.steps, 1500), min(args.warmup, 20)
            r = time_reference(args.size, w, k, threads)
            line["cpu_baseline"] = {"value": round(r["mlups"], 2), "unit": "MLUPS", "cores": r["threads"],
                                    "kind": "reference",
                                    "sample": f"{args.size}^3 lattice, {w} warm-up + {k} timed steps of OpenLB "
                                              f"CPU_SIMD+OpenMP ({r['binary']}) on {cpu_model()}"}
        except Exception as exc:  # the baseline is reported, never required for the GPU number
            line["cpu_baseline"] = {"value": None, "unit": "MLUPS", "cores": None, "kind": "reference",
                                    "sample": f"unavailable: {exc}"}
    if line is not None:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
