"""Slab decomposition (lbx_slabs_*): a lattice cut along x into slabs, stepped with one face
exchange per step, gives the populations of the undivided lattice bit for bit -- periodic boxes,
a porous medium with halfway bounce-back links across the faces between slabs, a walled cavity
with a moving lid, and the channel with velocity and pressure boundary cells -- in every storage
form, with slab counts that do and do not divide the extent.  Statistics agree to FP64 rounding
(the slabs' partial sums are added in another order).  The GPU tests run every slab on device 0:
this run has one GPU; slabs on different devices take the same path plus a peer copy of each face
buffer.
"""
from __future__ import annotations

import numpy as np
import pytest

import lbcases as L
from openlb_b200 import configs, lbx


def _random_pops(q, n, seed, scale=1e-3):
    rng = np.random.default_rng(seed)
    return (rng.random((q, n)) - 0.5) * scale


@pytest.mark.gpu
@pytest.mark.parametrize("storage", ["f64", "f32", "f16dev", "bf16dev"])
@pytest.mark.parametrize("q,core,n_slabs,periodic", [
    (19, (20, 12, 10), 2, (1, 1, 1)),
    (19, (23, 9, 11), 3, (1, 1, 1)),
    (27, (17, 8, 9), 4, (1, 1, 1)),
    (19, (30, 10, 12), 2, (0, 1, 1)),
    (9, (30, 14, 1), 3, (1, 1, 0)),
])
def test_periodic_box_matches_the_undivided_lattice(storage, q, core, n_slabs, periodic):
    f0 = _random_pops(q, int(np.prod(core)), seed=q + n_slabs)
    whole = lbx.BlockLattice(q, core, periodic, storage)
    whole.define_dynamics("trt", omega=1.3, magic=0.25)
    whole.set_populations(f0)
    whole.collide_and_stream(9, statistics=True)
    want = whole.get_populations()
    st_want = whole.get_statistics()
    whole.close()
    with lbx.SlabLattice(q, core, periodic, storage, n_slabs) as sl:
        assert sum(sl.nx) == core[0] and sl.x0[0] == 0
        sl.define_dynamics("trt", omega=1.3, magic=0.25)
        sl.set_populations(f0)
        sl.collide_and_stream(9, statistics=True)
        got = sl.get_populations()
        st = sl.get_statistics()
    assert st["cells"] == st_want["cells"]
    if periodic[0]:
        assert np.array_equal(got, want)
        for k in ("average_rho", "average_energy", "max_u"):
            assert abs(st[k] - st_want[k]) <= 1e-13 * max(abs(st_want[k]), 1e-300)
    else:
        # without periodic x the populations entering across the outer x faces are the padding's
        # (no boundary condition there): compare the cells they cannot have reached in 9 steps
        inner = np.zeros(core, bool)
        inner[9:-9] = True
        assert inner.any()
        assert np.array_equal(got[:, inner.reshape(-1)], want[:, inner.reshape(-1)])


@pytest.mark.gpu
@pytest.mark.parametrize("name,n_slabs", [("porous_d3q19_fbgk_f64", 2), ("porous_d3q27_fsmag_f64", 3),
                                          ("porous_d2q9_trt_f64", 2), ("cavity_d3q19_bb_f64", 2),
                                          ("cavity_d2q9_bgk_f64", 3)])
@pytest.mark.parametrize("storage", ["f64", "f16dev"])
def test_links_across_slab_faces_match_the_undivided_lattice(name, n_slabs, storage):
    """Reference fixtures with halfway bounce-back links (resting and moving walls) whose solid
    neighbours lie across the faces between slabs."""
    fx = L.load_fixture(name)
    setup = L.case_setup(fx)
    q, core, per = setup["q"], tuple(setup["core"]), setup["periodic"]
    if core[0] < 2 * n_slabs:
        pytest.skip("too few planes")
    steps = fx["meta"]["steps"]
    from test_gpu_parity import make_lattice
    whole = make_lattice(setup, storage)
    whole.set_populations(np.asarray(fx["f0"], np.float64))
    whole.collide_and_stream(steps)
    want = whole.get_populations()
    whole.close()
    with lbx.SlabLattice(q, core, per, storage, n_slabs) as sl:
        sl.define_dynamics(L.GPU_DYN[setup["dyn"]], omega=setup["omega"], magic=setup["magic"],
                           smagorinsky=setup["cs"], force=setup["force"])
        if setup["cell_dyn"] is not None:
            cd = np.asarray(setup["cell_dyn"])
            sl.set_cell_dynamics(np.where(cd >= 3, 0, cd).astype(np.uint8))
        if setup["links"] is not None:
            cells, dirs, wall = setup["links"]
            sl.set_bouzidi_links(cells, dirs, wall)
        sl.set_populations(np.asarray(fx["f0"], np.float64))
        sl.collide_and_stream(steps)
        got = sl.get_populations()
    mask = L.fluid_mask(fx)
    assert np.array_equal(got[:, mask], want[:, mask])


@pytest.mark.gpu
@pytest.mark.parametrize("storage", ["f64", "f16dev"])
def test_channel_with_boundary_cells_matches_the_undivided_lattice(storage):
    extent = (40, 20, 18)
    whole, mat = configs.channel_sphere(storage, extent, 0.04, 6.0, 20.0, (14, 10, 9))
    whole.collide_and_stream(30, statistics=True)
    want = whole.get_populations()
    st_want = whole.get_statistics()
    whole.close()
    sl, _ = configs.channel_sphere(storage, extent, 0.04, 6.0, 20.0, (14, 10, 9), slabs=3)
    sl.collide_and_stream(30, statistics=True)
    got = sl.get_populations()
    st = sl.get_statistics()
    sl.close()
    fluid = np.isin(mat.reshape(-1), (1, 3, 4))
    assert np.array_equal(got[:, fluid], want[:, fluid])
    assert abs(st["average_rho"] - st_want["average_rho"]) <= 1e-13


@pytest.mark.gpu
def test_boundary_cells_next_to_a_slab_face_are_refused():
    extent = (12, 10, 10)
    mat = configs.channel_materials(extent, (6, 5, 5), 2.0)
    with lbx.SlabLattice(27, extent, (0, 0, 0), "f32", 2) as sl:
        sl.define_dynamics("bgk", omega=1.2)
        cells = np.array([6 * 100 + 5 * 10 + 5])  # x = 6: the first plane of slab 1
        with pytest.raises(lbx.LbxError, match="within two planes"):
            sl.set_boundary_cells(cells, [1], [lbx.NORMAL_FLAT], [[0, 1, 0]], [[0, 0, 0, 0]])
    assert mat.shape == extent


@pytest.mark.gpu
def test_const_rho_is_refused_on_slabs():
    with lbx.SlabLattice(19, (8, 6, 6), (1, 1, 1), "f64", 2) as sl:
        sl.define_dynamics("const_rho_bgk", omega=1.2)
        with pytest.raises(lbx.LbxError, match="ConstRhoBGK"):
            sl.collide_and_stream(1)


def test_slab_creation_checks_its_arguments():
    import ctypes as C
    h = C.c_void_p()
    core = (C.c_int32 * 3)(5, 4, 4)
    per = (C.c_int32 * 3)(1, 1, 1)
    assert lbx.lib.lbx_slabs_create(19, core, per, 1, 3, None, C.byref(h)) == -1  # fewer than 2 planes a slab
    assert lbx.lib.lbx_slabs_create(19, core, per, 1, 0, None, C.byref(h)) == -1
    assert lbx.lib.lbx_slabs_collide_and_stream(None, 1, 0) == -1
