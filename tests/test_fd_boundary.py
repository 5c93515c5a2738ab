"""Flat-face velocity / pressure boundaries (boundary::InterpolatedVelocity and
boundary::InterpolatedPressure): the discrete-normal helper against the reference's own list,
argument checking on the CPU, and on the GPU the channel fixtures beyond what the generic
fixture tests cover (every storage form, launch-shape independence, initial post-processing).

Tolerances: FP64 within 1e-13 of the oracle (the GPU computes the boundary cells' velocities
before rewriting any of them, the reference one cell after the other; the two orders give the
same values up to rounding), FP32 within 1e-5 relative L2 in velocity of the reference's FP64
run, the 16-bit forms within 1e-3.
"""
import numpy as np
import pytest

import lbcases as L
from openlb_b200 import lbx

CHANNELS = [n for n in L.fixture_names() if n.startswith("channel_")]


@pytest.mark.parametrize("name", CHANNELS)
def test_normals_from_materials_match_the_reference_list(name):
    fx = L.load_fixture(name)
    meta = fx["meta"]
    ext = tuple(meta["ext"][:2]) if meta["q"] == 9 else tuple(meta["ext"])
    mat = fx["mat"].reshape(ext)
    per = L.periodic_of(meta)
    fd = L.fd_boundaries(fx["bnd"])
    for material, kind in ((3, 1), (4, 2)):
        cells, dirs, orients = lbx.fd_boundaries_from_materials(mat, material, fluid=(1,), outside=(0, 2),
                                                                periodic=per[: mat.ndim])
        sel = fd["kinds"] == kind
        assert np.array_equal(cells, fd["cells"][sel])
        assert np.array_equal(dirs, fd["dirs"][sel]) and np.array_equal(orients, fd["orients"][sel])


def test_corner_cells_are_not_flat():
    mat = np.ones((6, 5), np.int32)
    mat[0, :] = 3
    mat[:, 0] = 3
    cells, dirs, orients = lbx.fd_boundaries_from_materials(mat, 3, outside=(0,), periodic=(False, False))
    # the x = 0 row and the y = 0 column meet at (0, 0), an external corner: left out
    assert sorted(cells.tolist()) == [1, 2, 3, 5, 10, 15, 20]  # the far ends of each side have no normal
    _, types, normals = lbx.discrete_normals(mat, 3, outside=(0,), periodic=(False, False))
    assert types[0] == lbx.NORMAL_EXTERNAL_CORNER and normals[0].tolist() == [-1, -1, 0]


@pytest.mark.gpu
def test_fd_boundary_arguments_are_checked():
    lat = lbx.BlockLattice(19, (8, 6, 5), (0, 1, 1), "f64")
    v = np.zeros((1, 4))
    with pytest.raises(lbx.LbxError):  # normal along a periodic axis
        lat.set_fd_boundaries([0], [1], [1], [-1], v)
    with pytest.raises(lbx.LbxError):  # needs two cells inward
        lat.set_fd_boundaries([7 * 30], [1], [0], [-1], v)
    with pytest.raises(lbx.LbxError):  # pressure needs rho > 0
        lat.set_fd_boundaries([0], [2], [0], [-1], v)
    with pytest.raises(lbx.LbxError):  # duplicate cell
        lat.set_fd_boundaries([0, 0], [1, 1], [0, 0], [-1, -1], np.zeros((2, 4)))
    lat.close()
    # a flat cell at the end of a face: its neighbour along y is a padding cell, which carries no
    # dynamics (u = 0), as the reference's overlap does
    walls = lbx.BlockLattice(19, (8, 6, 5), (0, 0, 1), "f64")
    walls.set_fd_boundaries([0], [1], [0], [-1], v)
    walls.close()


def _run(name, storage, steps=None, variant=None):
    from test_gpu_parity import make_lattice
    fx = L.load_fixture(name)
    setup = L.case_setup(fx)
    lat = make_lattice(setup, storage)
    if variant is not None:
        lat.set_launch_config(*variant)
    lat.set_populations(np.asarray(fx["f0"], np.float64))
    lat.collide_and_stream(fx["meta"]["steps"] if steps is None else steps)
    out = lat.get_populations()
    lat.close()
    return fx, setup, out


@pytest.mark.gpu
@pytest.mark.parametrize("storage,tol", [("f32", 1e-5), ("f16dev", 1e-3), ("bf16dev", 1e-2)])
def test_channel_reduced_precision_forms(storage, tol):
    fx, setup, out = _run("channel_d3q19_bgk_f64", storage)
    e = L.errors(19, out, fx["fS"], L.fluid_mask(fx))
    assert e["u_l2"] <= tol, e


@pytest.mark.gpu
@pytest.mark.parametrize("variant", [(0, 256, 1, 1), (1, 64, 4, 1), (2, 32, 8, 2)])
def test_channel_launch_shapes_agree_bitwise(variant):
    _, _, a = _run("channel_d3q19_trt_f64", "f64")
    _, _, b = _run("channel_d3q19_trt_f64", "f64", variant=variant)
    assert np.array_equal(a, b)


@pytest.mark.gpu
def test_channel_statistics_count_the_boundary_cells():
    from test_gpu_parity import run_gpu
    fx = L.load_fixture("channel_d2q9_bgk_f64")
    setup = L.case_setup(fx)
    _, stats = run_gpu(setup, fx["f0"], fx["meta"]["steps"], "f64")
    ref = fx["stats"][-1]
    assert stats["cells"] == int(np.isin(fx["mat"], (1, 3, 4)).sum())
    assert abs(stats["average_rho"] - ref[0]) <= 1e-12 * abs(ref[0])
    assert abs(stats["max_u"] - ref[2]) <= 1e-12 * abs(ref[2])
