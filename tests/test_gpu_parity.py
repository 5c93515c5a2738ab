"""Parity of the CUDA path (liblbx.so through the C ABI) with the reference and the oracle.

Tolerances (written here, per the parity contract):
  FP64   populations within 2e-12 of the largest population against the reference's FP64
         run (DISABLE_CSE build) and within 1e-13 against the oracle (same algebra, same
         rounding: no FMA contraction in the FP64 kernels).
  FP32   velocity relative L2 error <= 1e-5 against the FP64 oracle started from the same
         populations, and <= 3e-5 against the reference's own FP32 run (whose CSE kernels
         round in another order).
  Statistics (FP64 accumulation) within 1e-12 relative for FP64 storage.
"""
from __future__ import annotations

import numpy as np
import pytest

import lbcases as L
from openlb_b200 import lbx

pytestmark = pytest.mark.gpu

F64 = [n for n in L.fixture_names() if n.endswith("_f64")]
F32 = [n for n in L.fixture_names() if n.endswith("_f32")]


def make_lattice(setup: dict, storage: str) -> lbx.BlockLattice:
    lat = lbx.BlockLattice(setup["q"], setup["core"], setup["periodic"], storage)
    lat.define_dynamics(L.GPU_DYN[setup["dyn"]], omega=setup["omega"], magic=setup["magic"],
                        smagorinsky=setup["cs"], force=setup["force"])
    for k, prm in (setup.get("classes") or {}).items():
        lat.set_dynamics_class(k, omega=prm["omega"], magic=prm["magic"], smagorinsky=prm["cs"], force=prm["force"],
                               dynamics=L.GPU_DYN[prm["dyn"]] if prm.get("dyn") else None)
    if setup["cell_dyn"] is not None:
        # boundary cells (ids 3 and 4) are marked by their own setters below
        cd = setup["cell_dyn"]
        lat.set_cell_dynamics(np.where((cd == 3) | (cd == 4), 0, cd).astype(np.uint8))
    if setup["links"] is not None:
        lat.set_bouzidi_links(*setup["links"])
    if setup.get("bbv") is not None:
        b = setup["bbv"]
        lat.set_bounce_back_velocity(b["cells"], b["rho"], b["u"])
    if setup.get("fd") is not None:
        fd = setup["fd"]
        if "normals" in fd:
            lat.set_boundary_cells(fd["cells"], fd["kinds"], fd["types"], fd["normals"], fd["values"])
        else:
            lat.set_fd_boundaries(fd["cells"], fd["kinds"], fd["dirs"], fd["orients"], fd["values"])
    return lat


def run_gpu(setup: dict, f0: np.ndarray, steps, storage: str = "f64", statistics: bool = True):
    lat = make_lattice(setup, storage)
    lat.set_populations(np.asarray(f0, np.float64))
    chunks = steps if isinstance(steps, (list, tuple)) else [steps]
    for k in chunks:
        lat.collide_and_stream(k, statistics=statistics)
    out = lat.get_populations(np.float64)
    stats = lat.get_statistics() if statistics else None
    lat.close()
    return out, stats


def forced(setup):
    return setup["force"] if setup["dyn"] in ("fbgk", "fsmag") else None


@pytest.mark.parametrize("name", F64)
def test_fp64_matches_reference_and_oracle(name):
    fx = L.load_fixture(name)
    setup = L.case_setup(fx)
    steps = fx["meta"]["steps"]
    out, stats = run_gpu(setup, fx["f0"], steps, "f64")
    mask = L.fluid_mask(fx)
    e_ref = L.errors(setup["q"], out, fx["fS"], mask, forced(setup))
    assert e_ref["pop"] <= 2e-12, e_ref
    orc, ost = L.run_oracle(setup, fx["f0"], steps)
    e_orc = L.errors(setup["q"], out, orc, mask, forced(setup))
    # ConstRhoBGK couples every cell to the lattice's average density, an FP64 sum whose
    # parallel order differs from the oracle's sequential one in the last bits
    assert e_orc["pop"] <= (1e-12 if setup["dyn"] == "constrho" else 1e-13), e_orc
    ref = fx["stats"][-1]
    assert abs(stats["average_rho"] - ref[0]) <= 1e-12 * abs(ref[0])
    assert abs(stats["average_energy"] - ref[1]) <= 1e-12 * abs(ref[1]) + 1e-300
    assert abs(stats["max_u"] - ref[2]) <= 1e-12 * abs(ref[2]) + 1e-300
    assert stats["cells"] == L.counted_cells(fx)


@pytest.mark.parametrize("name", F32)
def test_fp32_matches_reference(name):
    fx = L.load_fixture(name)
    setup = L.case_setup(fx)
    steps = fx["meta"]["steps"]
    f0 = fx["f0"].astype(np.float64)
    out, _ = run_gpu(setup, fx["f0"].astype(np.float32), steps, "f32", statistics=False)
    mask = L.fluid_mask(fx)
    truth, _ = L.run_oracle(setup, f0, steps)
    e_truth = L.errors(setup["q"], out, truth, mask, forced(setup))
    assert e_truth["u_l2"] <= 1e-5, e_truth
    e_ref = L.errors(setup["q"], out, fx["fS"], mask, forced(setup))
    assert e_ref["u_l2"] <= 3e-5, e_ref


def test_fp64_is_bitwise_equal_to_oracle_bgk():
    """Same operation order, no FMA, IEEE division: identical bits."""
    fx = L.load_fixture("periodic_d3q19_bgk_f64")
    setup = L.case_setup(fx)
    out, _ = run_gpu(setup, fx["f0"], 20, "f64")
    orc, _ = L.run_oracle(setup, fx["f0"], 20)
    assert np.array_equal(out, orc), np.abs(out - orc).max()


@pytest.mark.parametrize("name", ["periodic_d3q19_trt_f64", "cavity_d2q9_bgk_f64", "porous_d3q27_fsmag_f64"])
def test_split_calls_equal_one_call(name):
    fx = L.load_fixture(name)
    setup = L.case_setup(fx)
    steps = fx["meta"]["steps"]
    a, _ = run_gpu(setup, fx["f0"], steps)
    b, _ = run_gpu(setup, fx["f0"], [steps // 3, steps - steps // 3])
    assert np.array_equal(a, b)


EDGE = [(19, (1, 1, 1)), (19, (1, 3, 2)), (27, (3, 1, 1)), (27, (2, 2, 5)), (9, (1, 1, 1)), (9, (5, 1, 1)),
        (19, (33, 5, 40)), (27, (7, 9, 65)), (9, (70, 3, 1))]


@pytest.mark.parametrize("q,core", EDGE)
@pytest.mark.parametrize("dyn", ["bgk", "fsmag"])
def test_periodic_edge_shapes_match_oracle(q, core, dyn):
    rng = np.random.default_rng(q * 1000 + sum(core))
    n = int(np.prod(core))
    f0 = (rng.random((q, n)) - 0.5) * 0.05 * L.W[q][:, None]
    per = (1, 1, 1 if q != 9 else 0)
    setup = {"q": q, "core": core, "periodic": per, "dyn": dyn, "omega": 1.6, "magic": 0.25, "cs": 0.15,
             "force": [2e-4, -1e-4, 3e-4], "links": None, "cell_dyn": None}
    out, _ = run_gpu(setup, f0, 9)
    orc, _ = L.run_oracle(setup, f0, 9)
    assert np.abs(out - orc).max() <= 1e-13 * np.abs(orc).max()


@pytest.mark.parametrize("q", [9, 19, 27])
def test_channel_periodic_in_x_with_bounce_back_walls(q):
    """Mixed periodicity: periodic along x, bounce-back dynamics on the y walls, body force."""
    core = (12, 7, 1) if q == 9 else (10, 7, 6)
    nx, ny, nz = core
    mat = np.ones(core, np.int32)
    mat[:, 0, :] = 4
    mat[:, -1, :] = 4
    rng = np.random.default_rng(q)
    n = nx * ny * nz
    f0 = (rng.random((q, n)) - 0.5) * 0.02 * L.W[q][:, None]
    cd = np.where(mat.reshape(-1) == 1, 1, 2).astype(np.uint8)
    setup = {"q": q, "core": core, "periodic": (1, 0, 1 if q != 9 else 0), "dyn": "fbgk", "omega": 1.2,
             "magic": 0.25, "cs": 0.1, "force": [1e-4, 0, 0], "links": None, "cell_dyn": cd}
    out, _ = run_gpu(setup, f0, 30)
    orc, _ = L.run_oracle(setup, f0, 30)
    mask = mat.reshape(-1) == 1
    assert np.abs(out[:, mask] - orc[:, mask]).max() <= 1e-13 * np.abs(orc[:, mask]).max()


@pytest.mark.parametrize("q", [9, 19, 27])
def test_ini_equilibrium(q):
    core = (9, 8, 1) if q == 9 else (6, 5, 7)
    n = int(np.prod(core))
    d = 2 if q == 9 else 3
    rng = np.random.default_rng(q)
    rho = 1 + 0.01 * rng.standard_normal(n)
    u = 0.05 * rng.standard_normal((d, n))
    lat = lbx.BlockLattice(q, core, (1, 1, 1), "f64")
    lat.ini_equilibrium(rho, u)
    f = lat.get_populations()
    c = L.VEL[q][:, :d]
    cu = c @ u
    usq = (u * u).sum(axis=0)
    w = L.W[q][:, None]
    feq = rho * w * (1 + 3 * cu + 4.5 * cu * cu - 1.5 * usq) - w
    assert np.abs(f - feq).max() <= 1e-15
    r2, u2 = lat.compute_moments()
    assert np.allclose(r2, rho, rtol=1e-13, atol=0) and np.allclose(u2, u, rtol=0, atol=1e-14)


@pytest.mark.parametrize("storage", ["f64", "f32"])
def test_reductions_match_numpy(storage):
    fx = L.load_fixture("porous_d3q19_fbgk_f64")
    setup = L.case_setup(fx)
    lat = make_lattice(setup, storage)
    lat.set_populations(fx["f0"])
    lat.collide_and_stream(5)
    f = lat.get_populations()
    q = setup["q"]
    mask = L.fluid_mask(fx)
    c = L.VEL[q]
    rho = f[:, mask].sum(axis=0) + 1
    j = c.T @ f[:, mask]
    mm = lat.reduce(lbx.REDUCE_MASS_MOMENTUM)
    tol = 1e-12 if storage == "f64" else 1e-6
    assert abs(mm[0] - rho.sum()) <= tol * rho.sum()
    assert np.allclose(mm[1:], j.sum(axis=1), rtol=0, atol=tol * rho.sum() * 1e-2)
    # momentum exchange over the links: sum c_k (f_k(x_b + c_k) + f_opp(k)(x_b)) with full populations
    cells, dirs, _ = setup["links"]
    nx, ny, nz = setup["core"]
    opp = L.opposite(q)
    X = cells // (ny * nz)
    Y = (cells // nz) % ny
    Z = cells % nz
    xs = (((X + c[dirs, 0]) % nx) * ny + (Y + c[dirs, 1]) % ny) * nz + (Z + c[dirs, 2]) % nz
    w = L.W[q]
    s = f[dirs, xs] + w[dirs] + f[opp[dirs], cells] + w[opp[dirs]]
    drag = (c[dirs] * s[:, None]).sum(axis=0)
    got = lat.reduce(lbx.REDUCE_DRAG)
    assert np.allclose(got, drag, rtol=1e-9 if storage == "f64" else 1e-4, atol=1e-12)
    # residual: first call measures against zero, second against the snapshot
    r1 = lat.reduce(lbx.REDUCE_RESIDUAL)
    _, u = lat.compute_moments()
    un = np.sqrt((u[:, mask] ** 2).sum())
    assert np.isclose(r1[1], un, rtol=1e-5)
    lat.collide_and_stream(1)
    r2 = lat.reduce(lbx.REDUCE_RESIDUAL)
    _, u2 = lat.compute_moments()
    du = np.sqrt(((u2[:, mask] - u[:, mask].astype(np.float32)) ** 2).sum())
    assert np.isclose(r2[0], du, rtol=1e-4)
    lat.close()


def test_rotation_bookkeeping():
    lat = lbx.BlockLattice(19, (5, 6, 7), (1, 1, 1), "f32")
    info = lat.info()
    n = info.column_period
    sx, sy = info.padded[1] * info.padded[2], info.padded[2]
    lat.collide_and_stream(3)
    for i, c in enumerate(L.C19):
        off = c[0] * sx + c[1] * sy + c[2]
        assert lat.population_shift(i) == (-3 * off) % n
    lat.close()


def test_invalid_parameters_raise():
    lat = lbx.BlockLattice(19, (4, 4, 4), (1, 1, 1), "f32")
    with pytest.raises(lbx.LbxError):
        lat.define_dynamics("bgk", omega=2.5)
    with pytest.raises(lbx.LbxError):
        lat.set_cell_dynamics(np.full(64, 7, np.uint8))
    with pytest.raises(lbx.LbxError):
        lat.set_bouzidi_links([0], [27])
    lat.close()


@pytest.mark.parametrize("name", ["periodic_d3q27_fsmag_f64", "cavity_d3q19_bb_f64", "porous_d3q19_fbgk_f64",
                                  "porous_d2q9_trt_f64", "tgv_d3q19_bgk_f32"])
@pytest.mark.parametrize("storage", ["f64", "f32", "f16dev", "bf16dev"])
def test_kernel_variants_agree_bitwise(name, storage):
    """Every step kernel variant and launch shape computes identical bits (variant 3 moves whole
    tiles with bulk copies; the 16-bit forms also with four cells per thread)."""
    fx = L.load_fixture(name)
    setup = L.case_setup(fx)
    outs = []
    shapes = [(0, 256, 1, 1), (1, 64, 4, 1), (1, 32, 8, 1), (2, 32, 8, 1), (2, 64, 4, 2), (2, 256, 1, 1),
              (3, 256, 1, 1), (4, 256, 1, 1), (5, 128, 1, 1)]
    if storage in ("f16dev", "bf16dev"):
        shapes += [(2, 32, 4, 4), (2, 128, 1, 2)]
    for variant, bx, by, k in shapes:
        lat = make_lattice(setup, storage)
        lat.set_launch_config(variant, bx, by, k)
        lat.set_populations(np.asarray(fx["f0"], np.float64))
        lat.collide_and_stream(7)
        outs.append(lat.get_populations())
        lat.close()
    # cells without dynamics hold leftovers that never reach a fluid cell: the K-cells kernel
    # neither loads nor stores them, the others copy them across periodic faces
    mask = L.fluid_mask(fx)
    for o in outs[1:]:
        assert np.array_equal(outs[0][:, mask], o[:, mask])


@pytest.mark.parametrize("q,core,storage,k", [(19, (48, 64, 64), "f32", 1), (19, (48, 64, 256), "f16dev", 2),
                                              (27, (40, 48, 40), "f64", 1), (9, (700, 384, 1), "bf16dev", 2)])
def test_l2_prefetch_variant_matches_variant_2(q, core, storage, k):
    """Launch variant 5 (variant 2 plus the L2 bulk prefetch of the block one wave ahead) on
    lattices with several waves of blocks, so that the prefetch is issued: the same bits as
    variant 2 after 9 steps."""
    n = int(np.prod(core))
    rng = np.random.default_rng(q + k)
    f0 = (rng.random((q, n)) - 0.5) * 1e-3
    outs = []
    for variant in (2, 5):
        lat = lbx.BlockLattice(q, core, (1, 1, 1) if q != 9 else (1, 1, 0), storage)
        lat.define_dynamics("bgk", omega=1.4)
        lat.set_launch_config(variant, 128, 1, k)
        lat.set_populations(f0)
        lat.collide_and_stream(9)
        outs.append(lat.get_populations())
        lat.close()
    assert np.array_equal(outs[0], outs[1])


@pytest.mark.parametrize("name", ["periodic_d3q19_bgk_f64", "porous_d3q27_fsmag_f64", "cavity_d2q9_bgk_f64"])
def test_plain_and_doubled_column_mappings_agree(name, monkeypatch):
    """Columns mapped twice back to back (no wrap arithmetic) and one plain allocation (explicit
    wrap) give identical bits in every fluid cell."""
    fx = L.load_fixture(name)
    setup = L.case_setup(fx)
    out_d, _ = run_gpu(setup, fx["f0"], fx["meta"]["steps"])
    monkeypatch.setenv("LBX_PLAIN_COLUMNS", "1")
    lat = make_lattice(setup, "f64")
    info = lat.info()
    assert info.column_stride == info.column_period
    lat.close()
    out_p, _ = run_gpu(setup, fx["f0"], fx["meta"]["steps"])
    mask = L.fluid_mask(fx)  # solid cells carry period-dependent leftovers that never reach fluid
    assert np.array_equal(out_d[:, mask], out_p[:, mask])


def test_doubled_columns_are_used_by_default():
    lat = lbx.BlockLattice(19, (8, 8, 8), (1, 1, 1), "f32")
    info = lat.info()
    assert info.column_stride == 2 * info.column_period
    lat.close()


class _DeviceColumn:
    """A raw device array seen through __cuda_array_interface__ (only read here)."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False), "version": 2}


@pytest.mark.parametrize("storage,typestr", [("f64", "<f8"), ("f32", "<f4")])
def test_population_ptr_reaches_the_populations_in_place(storage, typestr):
    import torch
    rng = np.random.default_rng(5)
    core = (6, 5, 4)
    n = int(np.prod(core))
    lat = lbx.BlockLattice(19, core, (1, 1, 1), storage)
    lat.define_dynamics("bgk", omega=1.3)
    lat.set_populations((rng.random((19, n)) - 0.5) * 0.01)
    lat.collide_and_stream(3)
    want = lat.get_populations(np.float64)
    info = lat.info()
    sy, sz = info.padded[1] * info.padded[2], info.padded[2]
    x, y, z = np.unravel_index(np.arange(n), core)
    padded = (x + 1) * sy + (y + 1) * sz + z + 1
    for i in range(19):
        ptr, shift = lat.population_ptr(i)
        col = torch.as_tensor(_DeviceColumn(ptr, int(info.column_period), typestr), device="cuda").cpu().numpy()
        got = col[(padded + shift) % info.column_period]
        assert np.array_equal(got.astype(np.float64), want[i])
    lat.close()


@pytest.mark.parametrize("storage", ["f64", "f32", "f16dev"])
def test_parameter_classes_match_single_dynamics_lattices(storage):
    """Cells of a parameter class collide exactly as a lattice whose own parameters are the
    class's: a box split into two halves of different omega and force equals, cell for cell, the
    two lattices that carry one parameter set each where the halves do not interact yet (the
    first step), and a lattice whose every cell is class 2 equals one with those parameters."""
    rng = np.random.default_rng(5)
    core = (12, 10, 8)
    n = int(np.prod(core))
    f0 = (rng.random((19, n)) - 0.5) * 2e-3
    main = dict(omega=1.3, force=(1e-4, 0.0, 0.0))
    other = dict(omega=0.9, force=(0.0, -2e-5, 0.0))

    def run(setup_fn, steps):
        lat = lbx.BlockLattice(19, core, (1, 1, 1), storage)
        lat.define_dynamics("forced_bgk", **main)
        setup_fn(lat)
        lat.set_populations(f0)
        lat.collide_and_stream(steps, statistics=True)
        out = lat.get_populations()
        st = lat.get_statistics()
        lat.close()
        return out, st

    def all_class(lat):
        lat.set_dynamics_class(2, **other)
        lat.set_cell_dynamics(np.full(n, lbx.CELL_BULK_CLASS_2, np.uint8))

    def plain_other(lat):
        lat.define_dynamics("forced_bgk", **other)
        lat.set_launch_config(1, 128, 2, 1)

    got, st = run(all_class, 7)
    want, st_want = run(plain_other, 7)
    assert np.array_equal(got, want)
    for k in ("average_rho", "average_energy", "max_u"):
        assert abs(st[k] - st_want[k]) <= 1e-12 * abs(st_want[k])
    # half and half: after one step each cell of the class half equals the single-dynamics run
    half = np.zeros(core, np.uint8)
    half[: core[0] // 2] = 1
    half[core[0] // 2:] = lbx.CELL_BULK_CLASS_1

    def halves(lat):
        lat.set_dynamics_class(1, **other)
        lat.set_cell_dynamics(half.reshape(-1))

    mixed, _ = run(halves, 1)
    a, _ = run(lambda lat: lat.set_launch_config(1, 128, 2, 1), 1)
    inner_main = np.zeros(core, bool)
    inner_main[1: core[0] // 2 - 1] = True
    inner_other = np.zeros(core, bool)
    inner_other[core[0] // 2 + 1: -1] = True
    assert np.array_equal(mixed[:, inner_main.reshape(-1)], a[:, inner_main.reshape(-1)])
    assert np.array_equal(mixed[:, inner_other.reshape(-1)], want_1step(core, f0, storage, other)[:, inner_other.reshape(-1)])


def want_1step(core, f0, storage, params):
    lat = lbx.BlockLattice(19, core, (1, 1, 1), storage)
    lat.define_dynamics("forced_bgk", **params)
    lat.set_launch_config(1, 128, 2, 1)
    lat.set_populations(f0)
    lat.collide_and_stream(1)
    out = lat.get_populations()
    lat.close()
    return out


def test_parameter_class_arguments_are_checked():
    lat = lbx.BlockLattice(19, (8, 8, 8), (1, 1, 1), "f32")
    lat.define_dynamics("bgk", omega=1.2)
    with pytest.raises(lbx.LbxError):
        lat.set_dynamics_class(4, omega=1.0)
    with pytest.raises(lbx.LbxError):
        lat.set_dynamics_class(1, omega=2.5)
    lat.set_dynamics_class(1, omega=1.0)
    with pytest.raises(lbx.LbxError, match="variant 1"):
        lat.set_launch_config(2, 128, 1, 1)
    lat.set_dynamics_class(1, remove=True)
    lat.close()
