"""The ensemble engine (persistent kernel over many box cavities) against the single-lattice
path, the reference's cavity run, and itself (alone vs. in a mix).

Tolerances: the ensemble and the single-lattice kernels share the collision code and both are
built without implicit FMA contraction, so their FP32 moments agree bitwise; FP32 against the
reference's FP64 cavity run within 1e-5 relative L2 in velocity (the FP32 parity bound).
"""
import numpy as np
import pytest

import lbcases as L
from openlb_b200 import lbx

pytestmark = pytest.mark.gpu


def single_lattice_cavity(core, omega, ulid, steps, storage="f32", dynamics="bgk"):
    """The same cavity on the single-lattice path: a solid shell around the fluid, halfway
    bounce-back links, the top layer moving."""
    nx, ny, nz = core
    ext = (nx + 2, ny + 2, nz + 2)
    mat = np.full(ext, 2, np.int32)      # resting walls
    mat[1:-1, 1:-1, 1:-1] = 1            # fluid
    mat[:, -1, :] = 3                    # the whole top layer moves (edges included)
    lat = lbx.BlockLattice(19, ext, (0, 0, 0), storage)
    lat.define_dynamics(dynamics, omega=omega, magic=0.25)
    lat.set_cell_dynamics((mat.reshape(-1) == 1).astype(np.uint8))
    lat.set_bouzidi_boundary(mat, 1, (2, 3), [(0, 0, 0), (ulid, 0, 0)])
    lat.post_process()  # SuperLattice::initialize() applies the post-processors once
    lat.collide_and_stream(steps)
    rho, u = lat.compute_moments()
    lat.close()
    fluid = (mat.reshape(-1) == 1)
    return rho[fluid], u[:, fluid]


@pytest.mark.parametrize("dynamics", ["bgk", "trt"])
def test_ensemble_matches_single_lattice_bitwise(dynamics):
    core, omega, ulid, steps = (12, 10, 9), 1.3, 0.08, 150
    with lbx.Ensemble(19, "f32", slab_bytes=64 << 20, max_lattices=8) as ens:
        s = ens.admit(lbx.make_request(core, omega, ulid, tolerance=0.0, max_steps=10 ** 9, dynamics=dynamics))
        ens.run(steps)
        st = ens.statuses()[s]
        assert st[0] == lbx.SLOT_RUNNING and st[1] == steps
        rho_e, u_e = ens.moments(s)
    rho_s, u_s = single_lattice_cavity(core, omega, ulid, steps, dynamics=dynamics)
    assert np.array_equal(rho_e, rho_s) and np.array_equal(u_e, u_s)


def test_ensemble_matches_reference_cavity():
    fx = L.load_fixture("cavity_d3q19_bgk_f64")
    meta = fx["meta"]
    core = tuple(e - 2 for e in meta["ext"])
    with lbx.Ensemble(19, "f32", slab_bytes=64 << 20, max_lattices=4) as ens:
        s = ens.admit(lbx.make_request(core, meta["omega"], meta["ulid"], tolerance=0.0, max_steps=10 ** 9))
        ens.run(meta["steps"])
        _, u = ens.moments(s)
    fluid = L.fluid_mask(fx)
    _, u_ref = L.moments(19, fx["fS"][:, fluid])
    err = np.sqrt(((u - u_ref) ** 2).sum() / (u_ref ** 2).sum())
    assert err <= 1e-5, err


def test_result_is_the_same_alone_and_in_the_mix():
    """Continuous batching: a request's result does not depend on what else runs, nor on when
    the others were admitted."""
    a = lbx.make_request((16, 14, 12), 1.2, 0.05, tolerance=0.0, max_steps=10 ** 9)
    with lbx.Ensemble(19, "f32", slab_bytes=256 << 20, max_lattices=16) as alone:
        sa = alone.admit(a)
        alone.run(120)
        alone.run(80)
        ref_rho, ref_u = alone.moments(sa)
    with lbx.Ensemble(19, "f32", slab_bytes=256 << 20, max_lattices=16) as mix:
        mix.admit(lbx.make_request((32, 32, 32), 1.7, 0.1, tolerance=0.0, max_steps=10 ** 9))
        sa = mix.admit(a)
        mix.admit(lbx.make_request((9, 40, 7), 1.9, 0.02, tolerance=0.0, max_steps=10 ** 9, dynamics="trt"))
        mix.run(120)
        late = mix.admit(lbx.make_request((24, 24, 24), 1.5, 0.05, tolerance=0.0, max_steps=10 ** 9))
        mix.run(80)
        rho, u = mix.moments(sa)
        st = mix.statuses()
        assert st[sa][1] == 200 and st[late][1] == 80
    assert np.array_equal(rho, ref_rho) and np.array_equal(u, ref_u)


def test_convergence_retires_and_frees_the_slot():
    with lbx.Ensemble(19, "f32", slab_bytes=64 << 20, max_lattices=4) as ens:
        ens.set_config(threads=128, blocks_per_sm=0, check_interval=50)
        fast = ens.admit(lbx.make_request((8, 8, 8), 1.0, 0.05, tolerance=1e-4, max_steps=100000))
        capped = ens.admit(lbx.make_request((10, 10, 10), 1.9, 0.05, tolerance=1e-12, max_steps=300))
        for _ in range(40):
            ens.run(100)
            st = ens.statuses()
            if st[fast][0] != lbx.SLOT_RUNNING and st[capped][0] != lbx.SLOT_RUNNING:
                break
        assert st[fast][0] == lbx.SLOT_CONVERGED and st[fast][1] % 50 == 0 and st[fast][2] < 1e-4
        assert st[capped][0] == lbx.SLOT_MAX_STEPS and st[capped][1] == 300
        ens.run(100)
        assert ens.statuses()[fast][1] == st[fast][1]  # a finished lattice is not stepped
        ens.retire(fast)
        assert ens.statuses()[fast][0] == lbx.SLOT_FREE


def test_admission_by_footprint():
    big = lbx.make_request((96, 96, 96), 1.5, 0.05)
    with lbx.Ensemble(19, "f32", slab_bytes=100 << 20, max_lattices=8) as ens:
        fp = ens.footprint(big)
        assert 70 << 20 < fp < 100 << 20
        s = ens.admit(big)
        assert s is not None
        assert ens.admit(big) is None  # no room until the first one retires
        small = ens.admit(lbx.make_request((32, 32, 32), 1.5, 0.05))
        assert small is not None
        ens.retire(s)
        assert ens.admit(big) is not None


def test_divergence_is_detected_without_fault():
    with lbx.Ensemble(19, "f32", slab_bytes=64 << 20, max_lattices=4) as ens:
        ens.set_config(threads=256, blocks_per_sm=0, check_interval=20)
        bad = ens.admit(lbx.make_request((16, 16, 16), 1.999, 0.39, tolerance=0.0, max_steps=10 ** 9))
        ok = ens.admit(lbx.make_request((16, 16, 16), 1.2, 0.05, tolerance=0.0, max_steps=10 ** 9))
        for _ in range(30):
            ens.run(100)
            if ens.statuses()[bad][0] == lbx.SLOT_DIVERGED:
                break
        st = ens.statuses()
        assert st[bad][0] == lbx.SLOT_DIVERGED
        assert st[ok][0] == lbx.SLOT_RUNNING


def test_invalid_requests_are_refused():
    with lbx.Ensemble(19, "f32", slab_bytes=16 << 20, max_lattices=2) as ens:
        for req in (lbx.make_request((8, 8, 8), 2.5, 0.05), lbx.make_request((8, 8, 8), 1.5, float("nan")),
                    lbx.make_request((0, 8, 8), 1.5, 0.05)):
            with pytest.raises(lbx.LbxError):
                ens.admit(req)


def test_preempted_slot_resumes_exactly():
    """Pre-emption: a slot saved mid-run and restored into another ensemble (whose global step
    parity differs) continues bit for bit: populations, step count, residual and state."""
    r1 = lbx.make_request((16, 14, 12), 1.2, 0.05, tolerance=0.0, max_steps=10 ** 9)
    r2 = lbx.make_request((20, 18, 16), 1.7, 0.08, tolerance=1e-9, max_steps=10 ** 9, dynamics="trt")
    with lbx.Ensemble(19, "f32", slab_bytes=256 << 20, max_lattices=8) as a, \
            lbx.Ensemble(19, "f32", slab_bytes=256 << 20, max_lattices=8) as b:
        a.set_config(threads=128, blocks_per_sm=0, check_interval=50)
        b.set_config(threads=256, blocks_per_sm=0, check_interval=50)
        a.admit(r1)
        s2 = a.admit(r2)
        a.run(150)
        ckpt = a.save_slot(s2)
        a.run(120)
        want_status = a.statuses()[s2]
        want = a.moments(s2)
        other = b.admit(lbx.make_request((10, 10, 10), 1.5, 0.05, tolerance=0.0, max_steps=10 ** 9))
        b.run(37)
        s = b.restore_slot(ckpt)
        assert s != other
        assert b.statuses()[s][1] == 150
        b.run(120)
        assert b.statuses()[s] == want_status
        got = b.moments(s)
        assert all(np.array_equal(x, y) for x, y in zip(got, want))
        assert b.statuses()[other][1] == 157
        with pytest.raises(lbx.LbxError, match="checkpoint"):
            b.restore_slot(ckpt[:100])
    with lbx.Ensemble(19, "f64", slab_bytes=64 << 20, max_lattices=2) as c:
        with pytest.raises(lbx.LbxError, match="checkpoint"):
            c.restore_slot(ckpt)  # another storage form
