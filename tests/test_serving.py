"""The continuous-batching server: every request retires with a latency record, and each result is
the same whether the request ran alone or in the mix (admitted at whatever time its arrival and the
free memory allowed, next to whatever else was running).

Tolerance: bitwise.  A lattice's update does not read any other lattice's data and its residual is
summed over its own tiles in a fixed order, so neither the neighbours nor the admission time can
change its numbers; the FP32 moments of the same request alone and in the mix must be identical.
"""
import math

import numpy as np
import pytest

from openlb_b200 import serving


def test_sample_requests_is_seeded_and_follows_the_sweep():
    a = serving.sample_requests(400, seed=3)
    b = serving.sample_requests(400, seed=3)
    assert [(r.edge, r.reynolds, r.arrival) for r in a] == [(r.edge, r.reynolds, r.arrival) for r in b]
    edges = {r.edge for r in a}
    assert edges == {32, 48, 64, 96, 128, 192}
    re = np.array([r.reynolds for r in a])
    assert re.min() >= 10 and re.max() <= 1000
    assert abs(np.log(re).mean() - 0.5 * (np.log(10) + np.log(1000))) < 0.3
    gaps = np.diff([r.arrival for r in a])
    assert np.all(gaps >= 0) and abs(gaps.mean() - 1 / 200) < 0.002
    r = a[0]
    assert math.isclose(r.viscosity, 0.05 * r.edge / r.reynolds)
    assert 0 < r.omega < 2


def test_summary_statistics():
    recs = [serving.Record(i, 1000, arrival=0.0, finished=float(i + 1), steps=100, state=2) for i in range(100)]
    s = serving.summarise(recs, wall_seconds=100.0)
    assert s["requests"] == 100 and s["states"]["converged"] == 100
    assert s["p50_s"] == pytest.approx(50.5) and s["p99_s"] == pytest.approx(99.01)
    assert s["mlups"] == pytest.approx(100 * 1000 * 100 / 100 / 1e6)


@pytest.mark.gpu
def test_server_results_are_the_same_alone_and_in_the_mix():
    from openlb_b200 import lbx
    reqs = serving.sample_requests(14, seed=11, rate=2000.0, edges=(8, 12, 16, 20), re_range=(5, 60),
                                   tolerance=1e-5, max_steps=1500)
    reqs[3].max_steps = 70  # capped mid-chunk: retired with MAX_STEPS
    # A slab that holds only a few of them at a time, so admission waits for retirements.
    with lbx.Ensemble(19, "f32", slab_bytes=3 << 20, max_lattices=6) as ens:
        ens.set_config(threads=256, blocks_per_sm=0, check_interval=50)
        mix = serving.EnsembleServer(ens, chunk=100).serve(reqs, realtime=False, keep_fields=True)
    assert [r.rid for r in mix] == list(range(len(reqs)))
    assert max(r.admitted for r in mix) > min(r.finished for r in mix)  # later requests waited for a retirement
    for rec, req in zip(mix, reqs):
        assert rec.finished >= rec.admitted >= rec.arrival
        assert rec.state in (lbx.SLOT_CONVERGED, lbx.SLOT_MAX_STEPS)
        if rec.state == lbx.SLOT_CONVERGED:
            assert rec.residual < req.tolerance and rec.steps % 50 == 0
        else:
            assert rec.steps == req.max_steps
    assert mix[3].state == lbx.SLOT_MAX_STEPS and mix[3].steps == 70
    for rec, req in zip(mix, reqs):
        with lbx.Ensemble(19, "f32", slab_bytes=3 << 20, max_lattices=1) as ens:
            ens.set_config(threads=256, blocks_per_sm=0, check_interval=50)
            alone = serving.EnsembleServer(ens, chunk=100).serve([req], realtime=False, keep_fields=True)[0]
        assert (alone.state, alone.steps, alone.residual) == (rec.state, rec.steps, rec.residual)
        assert np.array_equal(alone.extra["moments"][0], rec.extra["moments"][0])
        assert np.array_equal(alone.extra["moments"][1], rec.extra["moments"][1])


@pytest.mark.gpu
def test_sequential_baseline_agrees_with_the_ensemble():
    """The sequential plain solves stop at the same residual criterion; their FP32 velocity matches
    the ensemble's after the same number of steps (the two paths share the collision code)."""
    from openlb_b200 import lbx
    reqs = serving.sample_requests(3, seed=5, edges=(10, 14), re_range=(5, 30), tolerance=1e-4, max_steps=2000)
    seq = serving.solve_sequential(reqs, check_interval=50, keep_fields=True)
    with lbx.Ensemble(19, "f32", slab_bytes=8 << 20, max_lattices=4) as ens:
        ens.set_config(threads=256, blocks_per_sm=0, check_interval=50)
        ensm = serving.EnsembleServer(ens, chunk=50).serve(reqs, realtime=False, keep_fields=True)
    for a, b in zip(seq, ensm):
        assert a.state == lbx.SLOT_CONVERGED and b.state == lbx.SLOT_CONVERGED
        assert abs(a.steps - b.steps) <= 50
        if a.steps == b.steps:
            assert np.array_equal(a.extra["moments"][1], b.extra["moments"][1])
