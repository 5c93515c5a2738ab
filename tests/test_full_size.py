"""The benchmark configuration at its full size (D3Q19 256^3 periodic Taylor-Green vortex, u0 =
0.05, nu = 0.01), checked through size-independent properties, since no oracle run of 16.8 M
cells x 1000 steps fits a test:

  - mass is conserved: the FP64 sum of rho after 1000 steps equals the initial one to the
    storage's rounding (1e-6 relative for FP32);
  - the kinetic energy decays at the viscous rate of the initial Fourier mode, E(t) / E(0) =
    exp(-2 nu |k|^2 t) with |k|^2 = 3 (2 pi / 256)^2, within 1 % after 1000 steps (the 3D TGV is not
    an exact Navier-Stokes solution, so the nonlinear transfer is allowed that much);
  - the FP32, FP16 and BF16 storage forms against the FP64 run of the same 300 steps: velocity
    L2 <= 5e-5 (FP32), <= 1e-3 (FP16, the precision form's bound), <= 1e-2 (BF16).
"""
import numpy as np
import pytest

from openlb_b200 import lbx

pytestmark = pytest.mark.gpu

N = 256
NU = 0.01
OMEGA = 1.0 / (3 * NU + 0.5)
U0 = 0.05


def tgv(n=N):
    x = 2 * np.pi * np.arange(n) / n
    sx, cx = np.sin(x), np.cos(x)
    ux = U0 * sx[:, None, None] * cx[None, :, None] * cx[None, None, :]
    uy = -U0 * cx[:, None, None] * sx[None, :, None] * cx[None, None, :]
    return np.ones(n ** 3), np.stack([ux.reshape(-1), uy.reshape(-1), np.zeros(n ** 3)])


def lattice(storage):
    lat = lbx.BlockLattice(19, (N, N, N), (1, 1, 1), storage)
    lat.define_dynamics("bgk", omega=OMEGA)
    lat.ini_equilibrium(*tgv())
    return lat


def test_mass_and_energy_decay_at_full_size():
    lat = lattice("f32")
    m0 = lat.reduce(lbx.REDUCE_MASS_MOMENTUM)
    lat.collide_and_stream(1, statistics=True)
    e1 = lat.get_statistics()["average_energy"]
    lat.collide_and_stream(999, statistics=True)
    st = lat.get_statistics()
    m1 = lat.reduce(lbx.REDUCE_MASS_MOMENTUM)
    lat.close()
    assert st["cells"] == N ** 3
    assert abs(m1[0] - m0[0]) <= 1e-6 * m0[0]
    assert np.all(np.abs(m1[1:]) <= 1e-6 * m0[0])  # the vortex carries no net momentum
    k2 = 3 * (2 * np.pi / N) ** 2
    expected = np.exp(-2 * NU * k2 * 999)
    assert abs(st["average_energy"] / e1 / expected - 1) < 0.01, (st["average_energy"] / e1, expected)


# The precision bound for a 16-bit form is a velocity L2 error of 1e-3 against FP64.  FP16
# meets it.  BF16 does not: its 8-bit mantissa rounds each stored deviation to about 4e-3 of
# itself, and the TGV ends near 2e-3 to 3e-3; the test states that as an expected failure.
@pytest.mark.parametrize("storage,tol", [
    ("f32", 5e-5), ("f16dev", 1e-3),
    pytest.param("bf16dev", 1e-3, marks=pytest.mark.xfail(strict=True, reason="BF16 misses the 1e-3 bound")),
])
def test_storage_forms_against_fp64_at_full_size(storage, tol):
    ref = lattice("f64")
    ref.collide_and_stream(300)
    _, u64 = ref.compute_moments()
    ref.close()
    lat = lattice(storage)
    lat.collide_and_stream(300)
    _, u = lat.compute_moments()
    lat.close()
    err = np.sqrt(((u - u64) ** 2).sum() / (u64 ** 2).sum())
    assert err <= tol, err
