"""The C++ host layer (openlb_b200/platform/lbx.hpp) through its example program cavity3d, a
lid-driven cavity set up like OpenLB's examples: defineDynamics<BGK>, setParameter<OMEGA>,
setBouzidiBoundary, initialize, collideAndStream, getStatistics.  Without a device the program
fails loudly (no CPU fallback); on a B200 its FP64 statistics equal those of the same cavity
driven through the Python binding bit for bit (same kernels, same order)."""
import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

from openlb_b200 import lbx

EXE = Path(lbx.LIB_PATH).parent / "cavity3d"


def test_example_is_built_and_fails_loudly_without_a_device():
    assert EXE.exists(), "run python -m openlb_b200.build"
    if lbx.device_count() > 0:
        pytest.skip("a device is present")
    proc = subprocess.run([str(EXE), "8", "2"], capture_output=True, text=True, timeout=120)
    assert proc.returncode == 1
    assert "lbx_lattice_create" in proc.stderr and "device" in proc.stderr


def _python_cavity(n, steps, re, storage):
    e = n + 2
    u_lid = 0.05
    omega = 1.0 / (3.0 * (u_lid * n / re) + 0.5)
    mat = np.full((e, e, e), 2, np.int32)
    mat[1:-1, 1:-1, 1:-1] = 1
    mat[:, -1, :] = 3
    lat = lbx.BlockLattice(19, (e, e, e), (0, 0, 0), storage)
    lat.define_dynamics("bgk", omega=omega)
    lat.set_cell_dynamics((mat.reshape(-1) == 1).astype(np.uint8))
    lat.set_bouzidi_boundary(mat, 1, (2, 3), [(0, 0, 0), (u_lid, 0, 0)])
    lat.post_process()
    lat.collide_and_stream(steps, statistics=True)
    st = lat.get_statistics()
    mass = lat.reduce(lbx.REDUCE_MASS_MOMENTUM)[0]
    lat.close()
    return st, mass, omega


@pytest.mark.gpu
@pytest.mark.parametrize("storage,arg", [("f64", "f64"), ("f32", "f32"), ("f16dev", "f16")])
def test_example_equals_the_python_binding(storage, arg):
    proc = subprocess.run([str(EXE), "20", "150", arg, "80"], capture_output=True, text=True, timeout=300)
    assert proc.returncode == 0, proc.stderr
    got = json.loads(proc.stdout.strip().splitlines()[-1])
    st, mass, omega = _python_cavity(20, 150, 80.0, storage)
    assert got["omega"] == omega
    assert got["cells"] == st["cells"] == 20 ** 3
    assert got["average_rho"] == st["average_rho"]
    assert got["average_energy"] == st["average_energy"]
    assert got["max_u"] == st["max_u"]
    assert got["mass"] == mass
    assert 0 < got["max_u"] < 0.1


EXE2 = Path(lbx.LIB_PATH).parent / "cavity2d"


def test_cavity2d_example_is_built_and_fails_loudly_without_a_device():
    assert EXE2.exists(), "run python -m openlb_b200.build"
    if lbx.device_count() > 0:
        pytest.skip("a device is present")
    proc = subprocess.run([str(EXE2), "14", "12", "2"], capture_output=True, text=True, timeout=120)
    assert proc.returncode == 1
    assert "lbx_lattice_create" in proc.stderr


@pytest.mark.gpu
def test_cavity2d_example_matches_the_reference():
    """cavity2d's set-up through the C++ layer -- defineDynamics<BGK> over material 1,
    boundary::set<InterpolatedVelocity> over the walls (2) and the lid (3, corners included),
    iniEquilibrium at rest, initialize() -- against the reference's own run of that set-up (the
    fixture geo_cavity2d_d2q9_ivel_bgk_rest_f64: 34 x 34, omega 1.6, lid 0.1, 400 steps)."""
    import lbcases as L
    fx = L.load_fixture("geo_cavity2d_d2q9_ivel_bgk_rest_f64")
    meta = fx["meta"]
    proc = subprocess.run([str(EXE2), "34", "34", str(meta["steps"]), "f64", repr(meta["omega"]), repr(meta["ulid"])],
                          capture_output=True, text=True, timeout=300)
    assert proc.returncode == 0, proc.stderr
    got = json.loads(proc.stdout.strip().splitlines()[-1])
    ref = fx["stats"][-1]
    assert got["cells"] == L.counted_cells(fx)
    assert abs(got["average_rho"] - ref[0]) <= 1e-12 * abs(ref[0])
    assert abs(got["average_energy"] - ref[1]) <= 1e-12 * abs(ref[1])
    assert abs(got["max_u"] - ref[2]) <= 1e-12 * abs(ref[2])
