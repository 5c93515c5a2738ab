"""The larger benchmark configurations as runnable set-ups (the GPU path only).

Channel past a sphere (default 512 x 128 x 128, D3Q27, TRT with magic 1/4): a sphere of
diameter 24 at (128, 64, 64) with halfway bounce-back, uniform inflow 0.04 through a flat
InterpolatedVelocity face at x = 0, an InterpolatedPressure face at the far end, periodic across
the section, Re = U d / nu = 50.

Porous medium (default 384^3, D3Q27, Smagorinsky-forced BGK with C_s = 0.12): non-overlapping
spheres of diameter U[8, 20] placed by seeded random sequential addition towards porosity 0.6,
periodic, body force F_x = 1e-6, nu = 0.05, halfway bounce-back on the sphere surfaces.

    python -m openlb_b200.configs channel --storage f16dev --steps 100
    python -m openlb_b200.configs porous --size 192 --steps 100
"""
from __future__ import annotations

import math
import time

import numpy as np

from . import lbx


def channel_sphere(storage: str = "f16dev", extent=(512, 128, 128), u_in: float = 0.04, d: int = 24,
                   re: float = 50.0) -> lbx.BlockLattice:
    """The channel lattice, initialised at the inflow velocity and post-processed once."""
    nx, ny, nz = extent
    nu = u_in * d / re
    omega = 1.0 / (3 * nu + 0.5)
    cx, cy, cz = nx // 4, ny // 2, nz // 2
    x, y, z = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    solid = (x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2 <= (d / 2) ** 2
    del x, y, z
    mat = np.where(solid, 2, 1).astype(np.int32)
    mat[0] = 3
    mat[-1] = 4
    lat = lbx.BlockLattice(27, (nx, ny, nz), (0, 1, 1), storage)
    lat.define_dynamics("trt", omega=omega, magic=0.25)
    lat.set_cell_dynamics(np.where(mat == 2, 0, 1).astype(np.uint8).reshape(-1))
    lat.set_bouzidi_boundary(mat, 1, (2,))
    n_face = ny * nz
    inlet = np.arange(n_face, dtype=np.int64)
    outlet = (nx - 1) * n_face + np.arange(n_face, dtype=np.int64)
    values = np.zeros((2 * n_face, 4))
    values[:n_face, 0] = u_in
    values[n_face:, 0] = 1.0
    lat.set_fd_boundaries(np.concatenate([inlet, outlet]), np.r_[np.ones(n_face), np.full(n_face, 2)],
                          np.zeros(2 * n_face), np.r_[-np.ones(n_face), np.ones(n_face)], values)
    u = np.zeros((3, nx * ny * nz))
    u[0] = np.where(mat.reshape(-1) == 2, 0.0, u_in)
    lat.ini_equilibrium(np.ones(nx * ny * nz), u)
    lat.post_process()
    return lat


def porous_spheres(n: int, seed: int = 7, porosity: float = 0.6, batches: int = 400, batch: int = 1000) -> np.ndarray:
    """Seeded random sequential addition of non-overlapping periodic spheres, d ~ U[8, 20]:
    candidates are drawn in batches and taken in order if they overlap neither an accepted
    sphere nor an earlier candidate of the batch (periodic distances), until the solid volume
    reaches 1 - porosity or the batches run out (the packing jams short of 0.6)."""
    from scipy.spatial import cKDTree
    rng = np.random.default_rng(seed)
    target = (1 - porosity) * n ** 3
    cen = np.zeros((0, 3))
    rad = np.zeros(0)
    filled = 0.0
    for _ in range(batches):
        if filled >= target:
            break
        c = rng.uniform(0, n, (batch, 3))
        r = rng.uniform(4, 10, batch)
        ok = np.ones(batch, bool)
        if len(cen):
            tree = cKDTree(cen, boxsize=n)
            for i, nbrs in enumerate(tree.query_ball_point(c, 20.0)):
                if nbrs:
                    dd = np.abs(cen[nbrs] - c[i])
                    dd = np.minimum(dd, n - dd)
                    if np.any((dd ** 2).sum(axis=1) < (rad[nbrs] + r[i]) ** 2):
                        ok[i] = False
        keep = []
        own = cKDTree(c, boxsize=n)
        for i in np.nonzero(ok)[0]:
            clash = False
            for j in own.query_ball_point(c[i], 20.0):
                if j in keep:
                    dd = np.abs(c[j] - c[i])
                    dd = np.minimum(dd, n - dd)
                    if (dd ** 2).sum() < (r[j] + r[i]) ** 2:
                        clash = True
                        break
            if not clash:
                keep.append(i)
                filled += 4 / 3 * math.pi * r[i] ** 3
                if filled >= target:
                    break
        cen = np.vstack([cen, c[keep]])
        rad = np.concatenate([rad, r[keep]])
    solid = np.zeros((n, n, n), bool)
    for c, r in zip(cen, rad):
        lo = np.floor(c - r).astype(int)
        hi = np.ceil(c + r).astype(int) + 1
        ix, iy, iz = (np.arange(lo[a], hi[a]) for a in range(3))
        X, Y, Z = np.meshgrid(ix, iy, iz, indexing="ij")
        inside = (X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2 <= r ** 2
        solid[np.ix_(ix % n, iy % n, iz % n)] |= inside
    return solid


def porous_medium(solid: np.ndarray, storage: str = "f16dev", nu: float = 0.05, force: float = 1e-6,
                  cs: float = 0.12) -> lbx.BlockLattice:
    n = solid.shape[0]
    mat = np.where(solid, 2, 1).astype(np.int32)
    lat = lbx.BlockLattice(27, (n, n, n), (1, 1, 1), storage)
    lat.define_dynamics("smagorinsky_forced_bgk", omega=1.0 / (3 * nu + 0.5), smagorinsky=cs, force=(force, 0, 0))
    lat.set_cell_dynamics(np.where(solid, 0, 1).astype(np.uint8).reshape(-1))
    lat.set_bouzidi_boundary(mat, 1, (2,))
    return lat


def main(argv=None) -> int:
    import argparse
    import json

    import torch

    ap = argparse.ArgumentParser(description="Run a benchmark configuration for a few steps and time it.")
    ap.add_argument("case", choices=["channel", "porous"])
    ap.add_argument("--storage", default="f16dev", choices=["f32", "f64", "f16dev", "bf16dev"])
    ap.add_argument("--size", type=int, nargs="+", help="channel: NX NY NZ; porous: N")
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--no-autotune", action="store_true")
    a = ap.parse_args(argv)
    if a.case == "channel":
        lat = channel_sphere(a.storage, tuple(a.size) if a.size else (512, 128, 128))
    else:
        lat = porous_medium(porous_spheres(a.size[0] if a.size else 384), a.storage)
    if not a.no_autotune:
        lat.autotune(steps=3)
    lat.collide_and_stream(2)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    lat.collide_and_stream(a.steps, statistics=True)
    st = lat.get_statistics()
    sec = time.perf_counter() - t0
    cells = lat.n_core
    lat.close()
    print(json.dumps({"case": a.case, "storage": a.storage, "cells": cells, "steps": a.steps,
                      "mlups": cells * a.steps / sec / 1e6, "statistics": st}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
