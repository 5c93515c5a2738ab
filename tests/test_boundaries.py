"""Velocity / pressure boundaries on flat faces, external edges and external corners, the
discrete-normal classifier and the boundary force, against the reference's own runs.

The "geo" fixtures come from the reference driver set up from a material map through the
reference's own setters (boundary::set<InterpolatedVelocity / InterpolatedPressure>, which
classify every cell with computeBoundaryTypeAndNormal; setBouzidiBoundary; the force functor
SuperLatticePhysBoundaryForce3D summed over the sphere).  test_oracle_golden and test_gpu_parity
run every fixture with the reference's own classification; the tests here add the library's
classifier, the path through the material-map setters, the boundary force and the Poiseuille
inlet profile.

Tolerances: classification exact; FP64 populations within 2e-12 of the largest population of the
reference run (the GPU reads the flat-face and edge densities it extrapolates from before the
priority-0 processors rewrite them, the reference one cell after the other: the two orders
differ by rounding only); boundary force within 1e-12 of |F| in FP64 and 1e-4 in FP32; FP32
velocity within 1e-5 relative L2 of the FP64 oracle.
"""
from __future__ import annotations

import numpy as np
import pytest

import lbcases as L

GEO = [n for n in L.fixture_names() if n.startswith("geo_")]
GEO64 = [n for n in GEO if n.endswith("_f64")]
FORCE = [n for n in GEO if "force" in np.load(L.GOLDEN / f"{n}.npz").files]


def _shape(meta):
    e = meta["ext"]
    return (int(e[0]), int(e[1])) if meta["q"] == 9 else (int(e[0]), int(e[1]), int(e[2]))


def test_local_boundary_fixtures_are_present():
    local = [n for n in GEO if "_lvel" in n]
    assert any("d2q9" in n for n in local) and any("d3q19" in n for n in local)
    assert any("lpres" in n for n in local)


def test_geo_fixtures_cover_edges_and_corners():
    kinds = set()
    for name in GEO:
        fx = L.load_fixture(name)
        kinds |= {(fx["meta"]["d"], int(t)) for t in fx["bclass"][:, 2]}
    assert (2, 0) in kinds and (2, 1) in kinds  # 2D flat faces and external corners
    assert (3, 0) in kinds and (3, 1) in kinds and (3, 3) in kinds  # 3D flat, corners, edges
    assert (2, 2) in kinds and (3, 2) in kinds and (3, 4) in kinds  # internal corners and edges
    assert any(n.startswith("geo_channel_d3q27_trt") for n in GEO)


@pytest.mark.parametrize("name", GEO)
def test_classifier_matches_the_reference(name):
    from openlb_b200 import lbx
    fx = L.load_fixture(name)
    meta = fx["meta"]
    a = L.geo_args(meta)
    mat = fx["mat"].reshape(_shape(meta))
    per = L.periodic_of(meta)[: mat.ndim]
    bc = fx["bclass"]
    for m, kind in [(m, 1) for m in a["ivel"] + a["ivel_lid"]] + [(m, 2) for m in a["ipres"]]:
        cells, types, normals = lbx.discrete_normals(mat, m, fluid=(1,), outside=(0,), periodic=per)
        rows = bc[(bc[:, 1] == kind) & np.isin(bc[:, 0], cells)]
        if kind == 2:  # the reference sets pressure conditions on flat faces only
            keep = types == 0
            cells, types, normals = cells[keep], types[keep], normals[keep]
        assert np.array_equal(rows[:, 0], cells)
        assert np.array_equal(rows[:, 2], types)
        assert np.array_equal(rows[:, 3:6], normals)


@pytest.mark.parametrize("name", [n for n in GEO if "channel" in n])
def test_poiseuille_profile_matches_the_reference(name):
    from openlb_b200 import configs
    fx = L.load_fixture(name)
    meta = fx["meta"]
    args = meta["args"]
    peak = float(args[args.index("--poiseuille") + 1])
    mat = fx["mat"].reshape(_shape(meta))
    u = configs.poiseuille_inlet(mat, 3, peak)
    ref = fx["vals"][:, :3].reshape(*mat.shape, 3)
    inlet = mat == 3
    # FP64: the same values; FP32: the reference evaluates the profile in float
    tol = 1e-15 if name.endswith("_f64") else 1e-8
    assert np.abs(u[inlet] - ref[inlet]).max() <= tol
    assert np.abs(u[inlet, 0]).max() <= peak


def _force_of(q, core, periodic, f, links_of_sphere):
    """BlockLatticePhysBoundaryForce3D summed over the sphere, from the populations of the core
    cells: F = sum over links (x_b, j) towards the sphere of c_j (f_opp(j)(x_b) + f_j(x_b + c_j))."""
    cells, dirs = links_of_sphere
    c = L.VEL[q]
    opp = L.opposite(q)
    nx, ny, nz = core
    x, y, z = cells // (ny * nz), (cells // nz) % ny, cells % nz
    xs = (x + c[dirs, 0]) % nx, (y + c[dirs, 1]) % ny, (z + c[dirs, 2]) % nz
    s_cell = (xs[0] * ny + xs[1]) * nz + xs[2]
    val = f[opp[dirs], cells] + f[dirs, s_cell]
    return (c[dirs].T * val).sum(axis=1)


@pytest.mark.parametrize("name", [n for n in FORCE if n.endswith("_f64")])
def test_oracle_force_matches_the_reference_functor(name):
    fx = L.load_fixture(name)
    meta = fx["meta"]
    setup = L.case_setup(fx)
    q, core = meta["q"], L.core_of(meta)
    a = L.geo_args(meta)
    mat = fx["mat"].reshape(core)
    cells, dirs, _ = L.bouzidi_links(q, core, mat, 1, a["force_mat"])
    rows = fx["force"]
    f = fx["f0"]
    step = 0
    for r in rows:
        f, _ = L.run_oracle(setup, f, int(r[0]) - step)
        step = int(r[0])
        got = _force_of(q, core, setup["periodic"], f, (cells, dirs))
        assert np.abs(got - r[1:4]).max() <= 1e-12 * np.abs(r[1:4]).max(), (r, got)


# ---- GPU ----------------------------------------------------------------------------------------
def build_from_materials(fx, storage):
    """The fixture's lattice set up the way an application would: bulk dynamics and cell map from
    the materials, halfway bounce-back from the materials, and the velocity / pressure boundaries
    through the library's own classifier (lbx_set_interpolated_boundary)."""
    from openlb_b200 import lbx
    meta = fx["meta"]
    a = L.geo_args(meta)
    q, core, per = meta["q"], L.core_of(meta), L.periodic_of(meta)
    mat = fx["mat"]
    lat = lbx.BlockLattice(q, core, per, storage)
    lat.define_dynamics(L.GPU_DYN[meta["dyn"]], omega=meta["omega"], magic=meta["magic"], smagorinsky=meta["cs"],
                        force=list(meta["force"]))
    cd = np.where(mat == 1, 1, 0).astype(np.uint8)
    for m in a["bounceback"]:
        cd[mat == m] = 2
    if a["bgk_mat"] is not None:  # BGK beside ForcedBGK: the forced dynamics with force 0
        other = None if meta["dyn"] in ("bgk", "fbgk") else "bgk"
        lat.set_dynamics_class(1, force=(0.0, 0.0, 0.0), dynamics=other)
        cd[mat == a["bgk_mat"]] = lbx.CELL_BULK_CLASS_1
    if a["trt_mat"] is not None:  # TRT beside another kind: a class of its own dynamics
        lat.set_dynamics_class(1, dynamics=None if meta["dyn"] == "trt" else "trt")
        cd[mat == a["trt_mat"]] = lbx.CELL_BULK_CLASS_1
    lat.set_cell_dynamics(cd)
    solid = list(a["bouzidi"]) + ([a["lid"]] if a["lid"] is not None else [])
    if solid:
        wall = None
        if a["lid"] is not None:
            wall = np.zeros((len(solid), 3))
            wall[-1, 0] = meta["ulid"]
        lat.set_bouzidi_boundary(mat, 1, solid, wall)
    if a["bbvel"]:
        cells = np.nonzero(np.isin(mat, a["bbvel"]))[0]
        lat.set_bounce_back_velocity(cells, fx["vals"][cells, 0], fx["vals"][cells, 1:4])
    vel, pres = (lbx.FD_VELOCITY, lbx.FD_PRESSURE)
    if a["local"]:
        vel, pres = ((lbx.FD_LOCAL_VELOCITY_RLB, lbx.FD_LOCAL_PRESSURE_RLB) if a["rlb"]
                     else (lbx.FD_LOCAL_VELOCITY, lbx.FD_LOCAL_PRESSURE))
    for m in a["ivel"] + a["ivel_lid"]:
        lat.set_interpolated_boundary(vel, mat, m, fx["vals"])
    for m in a["ipres"]:
        lat.set_interpolated_boundary(pres, mat, m, fx["vals"])
    return lat


@pytest.mark.gpu
@pytest.mark.parametrize("name", GEO64)
def test_material_setters_match_the_reference(name):
    fx = L.load_fixture(name)
    lat = build_from_materials(fx, "f64")
    lat.set_populations(np.asarray(fx["f0"], np.float64))
    lat.collide_and_stream(fx["meta"]["steps"])
    out = lat.get_populations()
    lat.close()
    setup = L.case_setup(fx)
    e = L.errors(fx["meta"]["q"], out, fx["fS"], L.fluid_mask(fx))
    assert e["pop"] <= 2e-12, e
    orc, _ = L.run_oracle(setup, fx["f0"], fx["meta"]["steps"])
    assert L.errors(fx["meta"]["q"], out, orc, L.fluid_mask(fx))["pop"] <= 1e-13
    if len(L.local_flat_cells(fx)):
        pops, cells = L.known_populations(fx)
        scale = np.abs(fx["fS"]).max()
        assert np.abs(out[pops, cells] - np.asarray(fx["fS"])[pops, cells]).max() <= 2e-12 * scale


@pytest.mark.gpu
@pytest.mark.parametrize("name", FORCE)
def test_boundary_force_matches_the_reference_functor(name):
    fx = L.load_fixture(name)
    meta = fx["meta"]
    a = L.geo_args(meta)
    storage = "f64" if name.endswith("_f64") else "f32"
    tol = 1e-12 if storage == "f64" else 1e-4
    lat = build_from_materials(fx, storage)
    group = a["bouzidi"].index(a["force_mat"][0])
    lat.set_populations(np.asarray(fx["f0"], np.float64))
    step = 0
    for r in fx["force"]:
        lat.collide_and_stream(int(r[0]) - step)
        step = int(r[0])
        got = lat.boundary_force(group)
        assert np.abs(got - r[1:4]).max() <= tol * np.abs(r[1:4]).max(), (r, got)
    lat.close()


@pytest.mark.gpu
@pytest.mark.parametrize("storage,tol", [("f32", 1e-5), ("f16dev", 1e-3)])
def test_edges_and_corners_in_reduced_precision(storage, tol):
    fx = L.load_fixture("geo_cavity_d3q19_ivel_bgk_f64")
    lat = build_from_materials(fx, storage)
    lat.set_populations(np.asarray(fx["f0"], np.float64))
    lat.collide_and_stream(fx["meta"]["steps"])
    out = lat.get_populations()
    lat.close()
    e = L.errors(19, out, fx["fS"], L.fluid_mask(fx))
    assert e["u_l2"] <= tol, e


@pytest.mark.gpu
@pytest.mark.parametrize("variant", [(0, 256, 1, 1), (1, 64, 4, 1), (2, 32, 8, 2), (3, 256, 1, 1)])
def test_edges_and_corners_launch_shapes_agree_bitwise(variant):
    fx = L.load_fixture("geo_cavity_d3q27_ivel_trt_f64")
    outs = []
    for v in (None, variant):
        lat = build_from_materials(fx, "f64")
        if v is not None:
            lat.set_launch_config(*v)
        lat.set_populations(np.asarray(fx["f0"], np.float64))
        lat.collide_and_stream(fx["meta"]["steps"])
        outs.append(lat.get_populations())
        lat.close()
    assert np.array_equal(outs[0], outs[1])


@pytest.mark.gpu
def test_boundary_cell_arguments_are_checked():
    from openlb_b200 import lbx
    lat = lbx.BlockLattice(19, (8, 6, 5), (0, 0, 0), "f64")
    v = np.zeros((1, 4))
    with pytest.raises(lbx.LbxError, match="two cells inward"):
        lat.set_boundary_cells([0], [1], [lbx.NORMAL_INTERNAL_CORNER], [[1, 1, 1]], v)
    with pytest.raises(lbx.LbxError, match="flat faces only"):
        lat.set_boundary_cells([0], [2], [lbx.NORMAL_INTERNAL_EDGE], [[-1, -1, 0]], np.array([[1.0, 0, 0, 0]]))
    with pytest.raises(lbx.LbxError, match="flat faces only"):
        v2 = np.array([[1.0, 0, 0, 0]])
        lat.set_boundary_cells([0], [2], [lbx.NORMAL_EXTERNAL_EDGE], [[-1, -1, 0]], v2)
    with pytest.raises(lbx.LbxError, match="normal type"):
        lat.set_boundary_cells([0], [1], [lbx.NORMAL_EXTERNAL_EDGE], [[-1, 0, 0]], v)
    with pytest.raises(lbx.LbxError, match="two cells inward"):
        lat.set_boundary_cells([0], [1], [lbx.NORMAL_EXTERNAL_CORNER], [[1, 1, 1]], v)
    lat.set_boundary_cells([0], [1], [lbx.NORMAL_EXTERNAL_CORNER], [[-1, -1, -1]], v)
    mat = np.ones((8, 6, 5), np.int32)
    mat[0] = 2
    with pytest.raises(lbx.LbxError, match="no discrete normal"):
        # a boundary layer with no fluid behind it at one cell: classify a lone boundary cell
        m2 = np.zeros((8, 6, 5), np.int32)
        m2[3, 3, 2] = 2
        lat.set_interpolated_boundary(lbx.FD_VELOCITY, m2, 2, np.zeros((8 * 6 * 5, 4)))
    lat.close()
