"""Continuous-batching request server over the ensemble engine, and the sequential baseline.

Parameter-sweep requests (lid-driven box cavities of different sizes and Reynolds numbers)
arrive over time.  `EnsembleServer.serve` admits every waiting request whose slab footprint
fits (skipping over ones that do not fit yet, so a large request does not block small ones
behind it), steps all admitted lattices together through one persistent launch per chunk of
steps, and retires each lattice as soon as the engine reports it converged (relative L2 velocity
residual below its tolerance), capped or diverged, freeing its slot and memory for the queue.
Requests that arrive while others are on the GPU join at the next chunk boundary.  The loop
itself is native (lbx_server_*, a host thread of the library); this module submits requests and
reads records.

`solve_sequential` solves the same requests one after another on the single-lattice path
(one lattice per launch sequence), the way a plain OpenLB run would.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import lbx


@dataclass
class CavityRequest:
    rid: int
    edge: int
    reynolds: float
    lid: float = 0.05
    tolerance: float = 1e-6
    max_steps: int = 50000
    arrival: float = 0.0  # seconds after the start of the run

    @property
    def viscosity(self) -> float:
        return self.lid * self.edge / self.reynolds

    @property
    def omega(self) -> float:
        return 1.0 / (3.0 * self.viscosity + 0.5)

    @property
    def cells(self) -> int:
        return self.edge ** 3

    def engine_request(self) -> lbx.EnsembleRequest:
        e = self.edge
        return lbx.make_request((e, e, e), self.omega, self.lid, self.tolerance, self.max_steps)


@dataclass
class Record:
    rid: int
    cells: int
    arrival: float
    admitted: float = math.nan
    finished: float = math.nan
    steps: int = 0
    state: int = 0
    residual: float = math.nan
    extra: dict = field(default_factory=dict)

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def sample_requests(n: int, seed: int = 0, rate: float = 200.0, edges=(32, 48, 64, 96, 128, 192),
                    re_range=(10.0, 1000.0), lid: float = 0.05, tolerance: float = 1e-6,
                    max_steps: int = 50000) -> list[CavityRequest]:
    """Seeded parameter sweep: edge uniform over `edges`, Re log-uniform over `re_range`,
    Poisson arrivals at `rate` per second."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, n)
    arrivals = np.cumsum(gaps) - gaps[0]
    es = rng.choice(np.asarray(edges), n)
    res = np.exp(rng.uniform(math.log(re_range[0]), math.log(re_range[1]), n))
    return [CavityRequest(i, int(es[i]), float(res[i]), lid, tolerance, max_steps, float(arrivals[i])) for i in range(n)]


def shard_requests(requests: list[CavityRequest], rank: int, world: int) -> list[CavityRequest]:
    """Requests of one rank when `world` GPUs serve one arrival stream: dealt round-robin in
    arrival order, so every rank sees the same rate and size mix and no request is served twice.
    The requests are independent, so the ranks need no collective on the data path."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    ordered = sorted(requests, key=lambda r: (r.arrival, r.rid))
    return ordered[rank::world]


class EnsembleServer:
    """Python driver of the native request loop (lbx.Server, include/lbx_server.h): submits the
    requests with their arrival times, lets the library's loop admit, step and retire them, and
    turns its records into Record objects.  `chunk` is the long run length; while a request
    waits for memory or is due to arrive, the loop runs `min_chunk` steps instead."""

    def __init__(self, ensemble: lbx.Ensemble, chunk: int = 500, stream=None, min_chunk: int | None = None):
        self.ens = ensemble
        self.chunk = chunk
        self.min_chunk = min(chunk, 100) if min_chunk is None else min_chunk
        self.stream = stream
        self.last_stats: dict = {}

    def serve(self, requests: list[CavityRequest], realtime: bool = True, keep_fields: bool = False) -> list[Record]:
        fields: dict[int, tuple] = {}
        errors: list[BaseException] = []

        def on_finish(rec) -> None:  # the loop's thread, before the slot is retired
            if rec.state not in (lbx.SLOT_CONVERGED, lbx.SLOT_MAX_STEPS, lbx.SLOT_DIVERGED):
                return
            try:
                rho = np.empty(rec.cells, np.float64)
                u = np.empty((3, rec.cells), np.float64)
                lbx.check(lbx.lib.lbx_ensemble_moments(self.ens._h, rec.slot, lbx._ptr(rho), lbx._ptr(u),
                                                       lbx._stream_ptr(self.stream)), "lbx_ensemble_moments")
                fields[rec.id] = (rho, u)
            except BaseException as e:  # reported after the loop ends
                errors.append(e)

        with lbx.Server(self.ens, self.min_chunk, self.chunk, realtime, self.stream,
                        on_finish if keep_fields else None) as srv:
            srv.submit((r.rid, r.arrival, r.engine_request()) for r in requests)
            srv.start()
            srv.close()
            srv.wait()
            raw = srv.records()
            self.last_stats = srv.stats()
        if errors:
            raise errors[0]
        records = []
        for d in raw:
            rec = Record(d["id"], d["cells"], d["arrival"], admitted=d["admitted"], finished=d["finished"],
                         steps=d["steps"], state=d["state"], residual=d["residual"])
            if keep_fields and d["id"] in fields:
                rec.extra["moments"] = fields[d["id"]]
            records.append(rec)
        return sorted(records, key=lambda r: r.rid)


def cavity_setup(edge: int, lid: float):
    """Host set-up of one cavity on the single-lattice path: the cell dynamics map (fluid core,
    no dynamics in the solid shell) and the halfway bounce-back links of the shell, the +y face
    moving with `lid`."""
    ext = (edge + 2, edge + 2, edge + 2)
    mat = np.full(ext, 2, np.int32)
    mat[1:-1, 1:-1, 1:-1] = 1
    mat[:, -1, :] = 3
    links = lbx.build_bouzidi_links(19, ext, mat, 1, (2, 3), [(0, 0, 0), (lid, 0, 0)])
    return ext, mat, (mat.reshape(-1) == 1).astype(np.uint8), links


def solve_sequential(requests: list[CavityRequest], check_interval: int = 100, storage: str = "f32",
                     device: int = 0, keep_fields: bool = False) -> list[Record]:
    """The same requests solved one at a time on the single-lattice path (cavity with a solid
    shell, halfway bounce-back links, residual checked every `check_interval` steps).  Each
    solve creates its lattice, as a plain program run does; the host set-up (cell map and link
    list) is derived once per cavity size and reused, so the baseline pays only the device side
    of the set-up per request."""
    records = []
    setups: dict[tuple[int, float], tuple] = {}
    t0 = time.perf_counter()
    for r in sorted(requests, key=lambda q: q.arrival):
        key = (r.edge, r.lid)
        if key not in setups:
            setups[key] = cavity_setup(r.edge, r.lid)
        ext, mat, cell_dyn, links = setups[key]
        rec = Record(r.rid, r.cells, r.arrival, admitted=time.perf_counter() - t0)
        with lbx.BlockLattice(19, ext, (0, 0, 0), storage, device=device) as lat:
            lat.define_dynamics("bgk", omega=r.omega)
            lat.set_cell_dynamics(cell_dyn)
            lat.set_bouzidi_links(*links)
            lat.post_process()
            steps, state, res = 0, lbx.SLOT_RUNNING, math.inf
            lat.reduce(lbx.REDUCE_RESIDUAL)  # snapshot of the initial velocity
            while state == lbx.SLOT_RUNNING:
                k = min(check_interval, r.max_steps - steps)
                lat.collide_and_stream(k)
                steps += k
                d, un, _ = lat.reduce(lbx.REDUCE_RESIDUAL)
                if k == check_interval:
                    res = d / un if un > 0 else (math.inf if d > 0 else 0.0)
                    if not math.isfinite(res) or not math.isfinite(un):
                        state = lbx.SLOT_DIVERGED
                    elif res < r.tolerance:
                        state = lbx.SLOT_CONVERGED
                if state == lbx.SLOT_RUNNING and steps >= r.max_steps:
                    state = lbx.SLOT_MAX_STEPS
            if keep_fields:
                rho, u = lat.compute_moments()
                fluid = mat.reshape(-1) == 1
                rec.extra["moments"] = (rho[fluid], u[:, fluid])
        rec.finished = time.perf_counter() - t0
        rec.steps, rec.state, rec.residual = steps, state, res
        records.append(rec)
    return records


def summarise(records: list[Record], wall_seconds: float) -> dict:
    lat = np.array([r.latency for r in records])
    updates = float(sum(r.cells * r.steps for r in records))
    states = {name: sum(1 for r in records if r.state == code) for name, code in
              (("converged", lbx.SLOT_CONVERGED), ("max_steps", lbx.SLOT_MAX_STEPS), ("diverged", lbx.SLOT_DIVERGED))}
    return {"requests": len(records), "wall_s": round(wall_seconds, 3),
            "mlups": round(updates / wall_seconds / 1e6, 1),
            "p50_s": round(float(np.percentile(lat, 50)), 4), "p99_s": round(float(np.percentile(lat, 99)), 4),
            "lattice_updates": updates, "states": states}


def time_ensemble(edges, steps: int, storage: str = "f32", mode: int = 1, cells: int = 2, threads: int = 256,
                  blocks_per_sm: int = 2, device: int = 0) -> dict:
    """Steps a fixed set of cavities (edge lengths `edges`, Re 100, no convergence stop) with one
    launch shape and returns the device-timed rate of the engine alone: one untimed run of
    `steps` steps (graph capture), then one timed run of `steps` steps."""
    import torch

    with lbx.Ensemble(19, storage, slab_bytes=8 << 30, max_lattices=max(8, len(edges)), device=device) as ens:
        ens.set_config(threads=threads, blocks_per_sm=blocks_per_sm, check_interval=100)
        ens.set_launch_mode(mode)
        ens.set_cells_per_thread(cells)
        for i, e in enumerate(edges):
            ens.admit(CavityRequest(i, e, 100.0, tolerance=0.0, max_steps=10 ** 9).engine_request())
        ens.run(steps)
        torch.cuda.synchronize(device)
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record()
        ens.run(steps)
        t1.record()
        torch.cuda.synchronize(device)
        ms = t0.elapsed_time(t1) / steps
    n = sum(e ** 3 for e in edges)
    return {"edges": list(edges), "storage": storage, "mode": mode, "cells_per_thread": cells, "threads": threads,
            "blocks_per_sm": blocks_per_sm, "ms_per_step": ms, "mlups": n / ms / 1e3}


def sweep(n: int, seed: int = 2024, max_steps: int = 50000, slab_gb: float = 24.0, sequential: bool = True,
          device: int = 0) -> dict:
    """The cavity parameter sweep as configured (edge ~ U{32..192}, Re log-uniform [10, 1000], lid
    0.05, Poisson arrivals at 200/s, residual < 1e-6 or `max_steps`), `n` requests of it: served by
    the ensemble server in real time, then (optionally) solved one after another."""
    import torch

    reqs = sample_requests(n, seed=seed, max_steps=max_steps)
    out: dict = {"requests": n, "seed": seed, "max_steps": max_steps, "slab_gb": slab_gb}
    with lbx.Ensemble(19, "f32", slab_bytes=int(slab_gb * (1 << 30)), max_lattices=512, device=device) as ens:
        ens.set_config(threads=256, blocks_per_sm=0, check_interval=100)
        probe = [ens.admit(CavityRequest(i, e, 100.0).engine_request()) for i, e in enumerate((32, 64, 128, 192))]
        ens.autotune(steps=10)
        for slot in probe:
            ens.retire(slot)
        server = EnsembleServer(ens, chunk=500, min_chunk=100)
        server.serve(sample_requests(4, seed=1, edges=(16,), max_steps=1000), realtime=False)
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        recs = server.serve(reqs)
        torch.cuda.synchronize(device)
        out["server"] = summarise(recs, time.perf_counter() - t0)
        out["server"]["loop"] = server.last_stats
        steps = np.array([r.steps for r in recs])
        out["server"]["steps_p50_p99_max"] = [int(np.percentile(steps, 50)), int(np.percentile(steps, 99)),
                                              int(steps.max())]
    if sequential:
        t0 = time.perf_counter()
        seq = solve_sequential(reqs, check_interval=100, device=device)
        torch.cuda.synchronize(device)
        out["sequential"] = summarise(seq, time.perf_counter() - t0)
        out["speedup_vs_sequential"] = round(out["sequential"]["wall_s"] / out["server"]["wall_s"], 3)
        same = [(a.state, a.steps) == (b.state, b.steps) for a, b in zip(recs, seq)]
        out["same_state_and_steps_as_sequential"] = f"{sum(same)}/{len(same)}"
    return out


def main(argv=None) -> int:
    import argparse
    import json

    ap = argparse.ArgumentParser(description="Time the ensemble engine on a fixed set of cavities.")
    ap.add_argument("--edges", default="192,128,96,64,48,32,128,96", help="comma-separated cavity edge lengths")
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--storage", default="f32", choices=["f32", "f64", "f16dev", "bf16dev"])
    ap.add_argument("--mode", type=int, default=1, help="0: persistent kernel, 1: graph of step launches")
    ap.add_argument("--cells", type=int, default=2, help="cells per thread (1 or 2)")
    ap.add_argument("--threads", type=int, default=256)
    ap.add_argument("--blocks-per-sm", type=int, default=2)
    ap.add_argument("--sweep", type=int, default=0,
                    help="serve this many requests of the cavity sweep as configured instead (50,000-step cap)")
    ap.add_argument("--max-steps", type=int, default=50000)
    ap.add_argument("--no-sequential", action="store_true")
    a = ap.parse_args(argv)
    if a.sweep:
        print(json.dumps(sweep(a.sweep, max_steps=a.max_steps, sequential=not a.no_sequential)))
        return 0
    edges = [int(v) for v in a.edges.split(",")]
    print(json.dumps(time_ensemble(edges, a.steps, a.storage, a.mode, a.cells, a.threads, a.blocks_per_sm)))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
