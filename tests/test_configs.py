"""The larger benchmark configurations at full size, run on the GPU path with their own physics
checks.  A reference oracle run of these sizes does not fit a test; the checks are stability,
conservation and the expected sign and order of the flow response.

Channel past a sphere (512 x 128 x 128, D3Q27, TRT with magic 1/4):
  - a sphere of diameter 24 at (128, 64, 64), halfway bounce-back;
  - uniform inflow 0.04 through a flat InterpolatedVelocity face at x = 0, an InterpolatedPressure
    face at x = 511, periodic across the section;
  - Re = U d / nu = 50, so nu = 0.0192;
  - FP16 and BF16 deviation storage.
  The reference's own setup has walls around the section, which needs the edge processors this
  build does not provide yet. The drag must be positive and finite, and the populations must stay
  finite.

Porous medium (384^3, D3Q27, Smagorinsky-forced BGK with C_s = 0.12, FP16):
  - non-overlapping spheres of diameter U[8, 20], placed by seeded random sequential addition
    towards porosity 0.6 (the addition jams near 0.70, which is what the test runs);
  - periodic, body force F_x = 1e-6, nu = 0.05 (the value this build records for the case);
  - halfway bounce-back on the sphere surfaces.
  Mass must be conserved and the mean x velocity must be positive, giving a finite permeability
  k = nu <u_x> / F_x.
"""
import math
import time

import numpy as np
import pytest

from openlb_b200 import lbx

pytestmark = pytest.mark.gpu


def _channel_sphere(storage, steps):
    nx, ny, nz = 512, 128, 128
    u_in, d, re = 0.04, 24, 50.0
    nu = u_in * d / re
    omega = 1.0 / (3 * nu + 0.5)
    x, y, z = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    solid = (x - 128) ** 2 + (y - 64) ** 2 + (z - 64) ** 2 <= (d / 2) ** 2
    mat = np.where(solid, 2, 1).astype(np.int32)
    mat[0] = 3
    mat[-1] = 4
    del x, y, z
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
    rho = np.ones(nx * ny * nz)
    u = np.zeros((3, nx * ny * nz))
    u[0] = np.where(mat.reshape(-1) == 2, 0.0, u_in)
    lat.ini_equilibrium(rho, u)
    lat.post_process()
    lat.collide_and_stream(1)
    lat.autotune(steps=3)
    import torch
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    lat.collide_and_stream(steps, statistics=True)
    st = lat.get_statistics()
    sec = time.perf_counter() - t0
    drag = lat.reduce(lbx.REDUCE_DRAG)
    lat.close()
    return st, drag, nx * ny * nz * steps / sec / 1e6


@pytest.mark.parametrize("storage", ["f16dev", "bf16dev"])
def test_channel_past_a_sphere_at_full_size(storage):
    st, drag, mlups = _channel_sphere(storage, 1000)
    print(f"channel-sphere 512x128x128 D3Q27 TRT {storage}: {mlups:.0f} MLUPS, drag {drag}, stats {st}")
    assert math.isfinite(st["average_rho"]) and math.isfinite(st["max_u"])
    assert 0.9 < st["average_rho"] < 1.1 and st["max_u"] < 0.2
    assert drag[0] > 0 and math.isfinite(drag[0])  # the flow pushes the sphere downstream
    assert abs(drag[1]) < 0.1 * drag[0] and abs(drag[2]) < 0.1 * drag[0]  # symmetric set-up


def _porous(n, seed=7, porosity=0.6, batches=400, batch=1000):
    """Seeded random sequential addition of non-overlapping periodic spheres, d ~ U[8, 20]:
    candidates are drawn in batches and taken in order if they overlap neither an accepted
    sphere nor an earlier candidate of the batch (periodic distances), until the solid volume
    reaches 1 - porosity or the batches run out (the packing jams short of 0.6 at these sizes)."""
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
                    d = np.abs(cen[nbrs] - c[i])
                    d = np.minimum(d, n - d)
                    if np.any((d ** 2).sum(axis=1) < (rad[nbrs] + r[i]) ** 2):
                        ok[i] = False
        keep = []
        own = cKDTree(c, boxsize=n)
        for i in np.nonzero(ok)[0]:
            clash = False
            for j in own.query_ball_point(c[i], 20.0):
                if j in keep:
                    d = np.abs(c[j] - c[i])
                    d = np.minimum(d, n - d)
                    if (d ** 2).sum() < (r[j] + r[i]) ** 2:
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


def test_porous_medium_at_full_size():
    n, nu, force, steps = 384, 0.05, 1e-6, 1000
    solid = _porous(n)
    porosity = 1 - solid.mean()
    mat = np.where(solid, 2, 1).astype(np.int32)
    lat = lbx.BlockLattice(27, (n, n, n), (1, 1, 1), "f16dev")
    lat.define_dynamics("smagorinsky_forced_bgk", omega=1.0 / (3 * nu + 0.5), smagorinsky=0.12, force=(force, 0, 0))
    lat.set_cell_dynamics(np.where(solid, 0, 1).astype(np.uint8).reshape(-1))
    lat.set_bouzidi_boundary(mat, 1, (2,))
    del mat
    m0 = lat.reduce(lbx.REDUCE_MASS_MOMENTUM)
    lat.autotune(steps=3)
    import torch
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    lat.collide_and_stream(steps, statistics=True)
    st = lat.get_statistics()
    sec = time.perf_counter() - t0
    m1 = lat.reduce(lbx.REDUCE_MASS_MOMENTUM)
    lat.close()
    ux = m1[1] / m1[0]  # mean x velocity over the fluid cells
    perm = nu * ux * porosity / force
    print(f"porous 384^3 D3Q27 Smagorinsky-forced FP16: porosity {porosity:.3f}, "
          f"{n ** 3 * steps / sec / 1e6:.0f} MLUPS, <u_x> {ux:.3e}, k = {perm:.3f}")
    assert 0.55 < porosity < 0.75
    assert abs(m1[0] - m0[0]) <= 1e-4 * m0[0]  # 16-bit storage: mass to the rounding of the form
    assert ux > 0 and math.isfinite(perm) and st["max_u"] < 0.1
