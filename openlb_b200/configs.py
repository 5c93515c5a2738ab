"""The larger benchmark configurations as runnable set-ups (the GPU path only).

Channel past a sphere (default 512 x 128 x 128, D3Q27, TRT with magic 1/4): a duct with
bounce-back side walls, a sphere of diameter 24 at (128, 64, 64) with halfway bounce-back,
a parabolic inflow (RectanglePoiseuille3D, peak 0.04) through an InterpolatedVelocity face at
x = 0 and an InterpolatedPressure face at the far end; Re = U_peak d / nu = 50.

Porous medium (default 384^3, D3Q27, Smagorinsky-forced BGK with C_s = 0.12): non-overlapping
spheres of diameter U[8, 20] placed by seeded random sequential addition (largest first) to
porosity 0.6, periodic, body force F_x = 1e-6, nu = 0.05, halfway bounce-back on the sphere
surfaces.

    python -m openlb_b200.configs channel --storage f16dev --steps 100
    python -m openlb_b200.configs porous --size 192 --steps 100
"""
from __future__ import annotations

import math
import time

import numpy as np

from . import lbx


def channel_materials(extent=(512, 128, 128), center=(128, 64, 64), d: float = 24) -> np.ndarray:
    """Material map of the channel past a sphere: walls (2) on the outer layer of the box, the
    inlet (3) and the outlet (4) on the interior of the x = 0 and x = end faces, the sphere (5):
    the fluid cells within d / 2 of `center`, fluid (1) elsewhere."""
    mat = np.full(extent, 2, np.int32)
    mat[1:-1, 1:-1, 1:-1] = 1
    mat[0, 1:-1, 1:-1] = 3
    mat[-1, 1:-1, 1:-1] = 4
    cx, cy, cz = center
    r2 = (d / 2) ** 2
    x = (np.arange(extent[0]) - cx)[:, None, None] ** 2
    y = (np.arange(extent[1]) - cy)[None, :, None] ** 2
    z = (np.arange(extent[2]) - cz)[None, None, :] ** 2
    mat[(x + y + z <= r2) & (mat == 1)] = 5
    return mat


def poiseuille_inlet(material: np.ndarray, inlet: int, peak: float) -> np.ndarray:
    """The inlet profile of RectanglePoiseuille3D over the cells of material `inlet` (functors/
    analytical/frameChangeF3D.hh:449-553): the zero-velocity planes lie half a cell outside the
    inlet's extent across the flow, and u = peak * 16 (d0/l0)(d1/l0)(d2/l1)(d3/l1) along the face
    normal, d0, d1 (d2, d3) the distances to the two planes of the first (second) cross axis and
    l0 = d0 + d1, l1 = d2 + d3.  Returns u[..., 3] over the whole map (zero off the inlet)."""
    cells = np.argwhere(material == inlet)
    lo, hi = cells.min(axis=0), cells.max(axis=0)
    normal = int(np.nonzero(lo == hi)[0][0])
    a1, a2 = [a for a in range(3) if a != normal]
    s1, e1 = lo[a1] - 0.5, hi[a1] + 0.5
    s2, e2 = lo[a2] - 0.5, hi[a2] + 0.5
    d0 = cells[:, a1] - s1
    d1 = e1 - cells[:, a1]
    d2 = cells[:, a2] - s2
    d3 = e2 - cells[:, a2]
    l0 = d0 + d1
    l1 = d2 + d3
    factor = 16.0 * d0 / l0 * d1 / l0 * d2 / l1 * d3 / l1
    u = np.zeros(material.shape + (3,))
    u[tuple(cells.T) + (np.zeros(len(cells), int),)] = peak * factor
    return u


def channel_sphere(storage: str = "f16dev", extent=(512, 128, 128), u_peak: float = 0.04, d: float = 24,
                   re: float = 50.0, center=None, rho_out: float = 1.0, slabs: int = 0):
    """The channel lattice at rest, post-processed once as SuperLattice::initialize does.
    D3Q27 TRT with magic 1/4, nu = u_peak d / Re; no-slip side walls of BounceBack dynamics
    (collision::Revert), halfway bounce-back on the sphere (link group 0);
    boundary::set<InterpolatedVelocity> on the inlet with the RectanglePoiseuille3D
    profile of peak u_peak along x, <InterpolatedPressure> with rho_out on the outlet.  Returns
    (lattice, material map); with slabs > 0 the lattice is a SlabLattice cut into that many
    slabs along x."""
    nx, ny, nz = extent
    if center is None:
        center = (nx // 4, ny // 2, nz // 2)
    nu = u_peak * d / re
    omega = 1.0 / (3 * nu + 0.5)
    mat = channel_materials(extent, center, d)
    if slabs:
        lat = lbx.SlabLattice(27, extent, (0, 0, 0), storage, slabs)
    else:
        lat = lbx.BlockLattice(27, extent, (0, 0, 0), storage)
    lat.define_dynamics("trt", omega=omega, magic=0.25)
    cell = np.zeros(mat.shape, np.uint8)
    cell[mat == 1] = lbx.CELL_BULK
    cell[mat == 2] = lbx.CELL_BOUNCE_BACK
    lat.set_cell_dynamics(cell.reshape(-1))
    lat.set_bouzidi_boundary(mat, 1, (5,))
    vals = np.zeros(mat.shape + (4,))
    vals[..., :3] = poiseuille_inlet(mat, 3, u_peak)
    vals[mat == 4, 0] = rho_out
    vals = vals.reshape(-1, 4)
    lat.set_interpolated_boundary(lbx.FD_VELOCITY, mat, 3, vals)
    lat.set_interpolated_boundary(lbx.FD_PRESSURE, mat, 4, vals)
    lat.post_process()
    return lat, mat


def drag_coefficient(force_x: float, u: float, d: float, rho: float = 1.0) -> float:
    """2 F_x / (rho u^2 A) with A = pi d^2 / 4, the frontal area of the sphere."""
    return 2.0 * force_x / (rho * u * u * math.pi * d * d / 4.0)


def porous_spheres(n: int, seed: int = 7, porosity: float = 0.6, d_min: float = 8.0, d_max: float = 20.0,
                   tries: int = 64, batch: int = 32) -> np.ndarray:
    """Seeded random sequential addition of non-overlapping spheres in a periodic n^3 box.

    Diameters are drawn uniformly from [d_min, d_max] until their volume is 1.3 times the solid
    volume wanted, then placed largest first: each sphere tries up to `tries` batches of `batch`
    uniform random centres and takes the first centre whose periodic distance to every placed
    sphere is at least the sum of the radii (a sphere that finds none is skipped).  Placing the
    large spheres first leaves the gaps to the small ones, which lets the addition pass the
    jamming point of drawing sizes in random order.  The solid cells are those whose centre lies
    in a sphere; the addition stops once they make up 1 - porosity of the box.  Returns the
    boolean solid map."""
    from scipy.spatial import cKDTree
    rng = np.random.default_rng(seed)
    target = (1 - porosity) * n ** 3
    diameters = []
    vol = 0.0
    while vol < 1.3 * target:
        d = rng.uniform(d_min, d_max)
        diameters.append(d)
        vol += math.pi * d ** 3 / 6
    diameters = np.sort(np.array(diameters))[::-1]
    cen = np.zeros((0, 3))
    rad = np.zeros(0)
    tree, in_tree = None, 0
    solid = np.zeros((n, n, n), bool)
    count = 0
    for d in diameters:
        r = d / 2
        for _ in range(tries):
            c = rng.uniform(0, n, (batch, 3))
            ok = np.ones(batch, bool)
            if tree is not None:  # spheres in the tree, within reach of a candidate
                for i, nb in enumerate(tree.query_ball_point(c, r + d_max / 2)):
                    if nb:
                        dd = np.abs(cen[nb] - c[i])
                        dd = np.minimum(dd, n - dd)
                        if np.any((dd ** 2).sum(axis=1) < (rad[nb] + r) ** 2):
                            ok[i] = False
            if in_tree < len(cen):  # spheres placed since the tree was built
                dd = np.abs(cen[None, in_tree:] - c[:, None])
                dd = np.minimum(dd, n - dd)
                ok &= ~np.any((dd ** 2).sum(axis=2) < (rad[None, in_tree:] + r) ** 2, axis=1)
            hit = np.nonzero(ok)[0]
            if len(hit) == 0:
                continue
            cc = c[hit[0]]
            cen = np.vstack([cen, cc])
            rad = np.append(rad, r)
            lo = np.floor(cc - r).astype(int)
            hi = np.ceil(cc + r).astype(int) + 1
            ix, iy, iz = (np.arange(lo[a], hi[a]) for a in range(3))
            inside = ((ix[:, None, None] - cc[0]) ** 2 + (iy[None, :, None] - cc[1]) ** 2
                      + (iz[None, None, :] - cc[2]) ** 2) <= r * r
            box = np.ix_(ix % n, iy % n, iz % n)
            count += int((inside & ~solid[box]).sum())
            solid[box] |= inside
            break
        if len(cen) - in_tree >= 256:
            tree, in_tree = cKDTree(cen, boxsize=n), len(cen)
        if count >= target:
            break
    return solid


def porous_medium(solid: np.ndarray, storage: str = "f16dev", nu: float = 0.05, force: float = 1e-6,
                  cs: float = 0.12, slabs: int = 0):
    """The porous box: Smagorinsky-forced BGK in the pores, no dynamics in the solid, halfway
    bounce-back links on every pore-solid face; a SlabLattice of `slabs` slabs when slabs > 0."""
    n = solid.shape[0]
    mat = np.where(solid, 2, 1).astype(np.int32)
    if slabs:
        lat = lbx.SlabLattice(27, (n, n, n), (1, 1, 1), storage, slabs)
    else:
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
        lat, _ = channel_sphere(a.storage, tuple(a.size) if a.size else (512, 128, 128))
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
