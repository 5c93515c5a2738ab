"""The project-written autotuners (lbx_autotune, lbx_ensemble_autotune): they time every launch
shape on the caller's own data, keep the fastest, and leave the state as it was, so a tuned run
continues bit for bit like an untuned one.  Tolerance: bitwise (every launch shape computes the
same bits: no implicit FMA contraction, residuals summed per 32-cell slot in a fixed order)."""
import numpy as np
import pytest

import lbcases as L
from openlb_b200 import lbx

pytestmark = pytest.mark.gpu


def _lattice(storage):
    lat = lbx.BlockLattice(19, (40, 24, 72), (1, 1, 1), storage)
    lat.define_dynamics("bgk", omega=1.6)
    rng = np.random.default_rng(7)
    lat.set_populations((rng.random((19, 40 * 24 * 72)) - 0.5) * 0.01 / 18)
    return lat


@pytest.mark.parametrize("storage", ["f32", "f16dev"])
def test_autotune_keeps_the_state_and_the_results(storage):
    tuned, plain = _lattice(storage), _lattice(storage)
    tuned.collide_and_stream(3)
    plain.collide_and_stream(3)
    before = tuned.get_populations()
    shifts = [tuned.population_shift(i) for i in range(19)]
    entries = tuned.autotune(steps=4)
    assert len(entries) >= 4
    timed = [e for e in entries if e["ms_per_step"] > 0]
    assert timed and {e["variant"] for e in timed} >= {0, 1, 2}
    assert np.array_equal(tuned.get_populations(), before)
    assert [tuned.population_shift(i) for i in range(19)] == shifts
    tuned.collide_and_stream(25)
    plain.collide_and_stream(25)
    assert np.array_equal(tuned.get_populations(), plain.get_populations())
    tuned.close()
    plain.close()


def test_autotune_with_bounce_back_links():
    """A tuned cavity with halfway bounce-back links still matches the reference's FP64 run."""
    from test_gpu_parity import make_lattice
    fx = L.load_fixture("cavity_d3q19_bgk_f64")
    setup = L.case_setup(fx)
    lat = make_lattice(setup, "f64")
    lat.set_populations(np.asarray(fx["f0"], np.float64))
    lat.autotune(steps=3)
    lat.collide_and_stream(fx["meta"]["steps"])
    out = lat.get_populations()
    lat.close()
    e = L.errors(setup["q"], out, fx["fS"], L.fluid_mask(fx), None)
    assert e["pop"] <= 2e-12, e


def _mix(ens):
    reqs = [lbx.make_request((20, 18, 16), 1.5, 0.05, tolerance=1e-5, max_steps=10 ** 6),
            lbx.make_request((33, 9, 40), 1.8, 0.08, tolerance=0.0, max_steps=10 ** 6, dynamics="trt"),
            lbx.make_request((7, 7, 7), 1.2, 0.02, tolerance=1e-3, max_steps=10 ** 6)]
    return [ens.admit(r) for r in reqs]


def test_ensemble_autotune_keeps_every_lattice_state():
    with lbx.Ensemble(19, "f32", slab_bytes=64 << 20, max_lattices=8) as tuned, \
            lbx.Ensemble(19, "f32", slab_bytes=64 << 20, max_lattices=8) as plain:
        for ens in (tuned, plain):
            ens.set_config(threads=256, blocks_per_sm=0, check_interval=40)
        st, sp = _mix(tuned), _mix(plain)
        tuned.run(120)
        plain.run(120)
        before = tuned.statuses()
        m_before = [tuned.moments(s) for s in st]
        entries = tuned.autotune(steps=30)
        assert any(e["ms_per_step"] > 0 for e in entries)
        assert {e["threads"] for e in entries} == {64, 128, 256}
        assert {e["variant"] for e in entries} == {0, 1}  # both launch modes tried
        assert {e["cells_per_thread"] for e in entries} == {1, 2}
        assert tuned.statuses() == before
        for s, (r0, u0) in zip(st, m_before):
            r1, u1 = tuned.moments(s)
            assert np.array_equal(r0, r1) and np.array_equal(u0, u1)
        tuned.run(300)
        plain.run(300)
        assert tuned.statuses() == plain.statuses()
        for a, b in zip(st, sp):
            ra, ua = tuned.moments(a)
            rb, ub = plain.moments(b)
            assert np.array_equal(ra, rb) and np.array_equal(ua, ub)


@pytest.mark.parametrize("threads,blocks,mode,cells,storage", [
    (64, 0, 0, 1, "f32"), (128, 2, 0, 1, "f32"), (256, 1, 0, 1, "f32"), (256, 0, 1, 1, "f32"), (64, 3, 1, 1, "f32"),
    (256, 0, 0, 2, "f32"), (128, 0, 1, 2, "f32"), (64, 5, 1, 2, "f32"), (256, 0, 1, 2, "f16dev"),
    (96, 0, 0, 2, "bf16dev"), (128, 0, 1, 2, "f64")])
def test_ensemble_results_do_not_depend_on_the_launch_shape(threads, blocks, mode, cells, storage):
    """Launch shape, launch mode (one persistent kernel, or one launch per step in a graph) and
    cells per thread give identical populations, step counts, states and residuals."""
    with lbx.Ensemble(19, storage, slab_bytes=64 << 20, max_lattices=8) as a, \
            lbx.Ensemble(19, storage, slab_bytes=64 << 20, max_lattices=8) as b:
        a.set_config(threads=256, blocks_per_sm=0, check_interval=40)
        b.set_config(threads=threads, blocks_per_sm=blocks, check_interval=40)
        b.set_launch_mode(mode)
        b.set_cells_per_thread(cells)
        sa, sb = _mix(a), _mix(b)
        a.run(200)
        b.run(200)
        assert a.statuses() == b.statuses()
        for x, y in zip(sa, sb):
            assert all(np.array_equal(p, q) for p, q in zip(a.moments(x), b.moments(y)))
