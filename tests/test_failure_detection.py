"""Failure detection without a GPU fault: the library's bounded waits are made to run out through
the test hook lbx_test_fault (off by default), and the status the caller reads is checked; an
allocation is made to fail the way cudaMalloc fails when memory is short; a running ensemble
request is cancelled between runs.  No test faults, traps or hangs the GPU: every wait that runs
out here is bounded (a few thousand polls), and the hook only leaves out an arrival or a copy.
"""
from __future__ import annotations

import numpy as np
import pytest

from openlb_b200 import lbx

pytestmark = pytest.mark.gpu

NONE, BARRIER, BULK, ALLOC = 0, 1, 2, 3


@pytest.fixture(autouse=True)
def _hook_off():
    lbx.lib.lbx_test_fault.argtypes = [lbx.C.c_int32, lbx.C.c_int32]
    lbx.lib.lbx_test_fault.restype = lbx.C.c_int
    yield
    assert lbx.lib.lbx_test_fault(NONE, 0) == 0


def _fault(kind, param):
    assert lbx.lib.lbx_test_fault(kind, param) == 0


def test_ensemble_grid_barrier_timeout_is_reported_and_the_context_stays_usable():
    with lbx.Ensemble(19, "f32", slab_bytes=256 << 20, max_lattices=8) as ens:
        ens.set_launch_mode(0)  # one persistent cooperative kernel with grid barriers
        slots = [ens.admit(lbx.make_request((16, 16, 16), 1.2, 0.05)) for _ in range(2)]
        assert None not in slots
        _fault(BARRIER, 20000)
        ens.run(10)
        with pytest.raises(lbx.LbxError, match="grid barrier"):
            ens.statuses()
        # hook off: the next run (another step count: a newly prepared launch) succeeds
        _fault(NONE, 0)
        ens.run(11)
        st = ens.statuses()
        assert all(s[0] == lbx.SLOT_RUNNING for s in st[:2])


def _bulk_lattice(f0):
    lat = lbx.BlockLattice(19, (32, 32, 32), (1, 1, 1), "f16dev")
    lat.define_dynamics("bgk", omega=1.5)
    lat.set_populations(f0)
    lat.set_launch_config(3, 256, 1, 1)
    return lat


def test_bulk_copy_wait_timeout_is_reported_and_the_lattice_stays_usable():
    rng = np.random.default_rng(3)
    f0 = (rng.random((19, 32 ** 3)) - 0.5) * 1e-3
    lat = _bulk_lattice(f0)
    _fault(BULK, 20000)
    lat.collide_and_stream(1, statistics=True)
    with pytest.raises(lbx.LbxError, match="gave up waiting"):
        lat.get_statistics()
    _fault(NONE, 0)
    # the error flag was cleared by the report; steps run again from a fresh state and give the
    # bits of a lattice that never saw the timeout
    lat.set_populations(f0)
    lat.collide_and_stream(3, statistics=True)
    st = lat.get_statistics()
    assert np.isfinite(st["average_rho"])
    got = lat.get_populations(np.float32)
    lat.close()
    ref = _bulk_lattice(f0)
    ref.collide_and_stream(3, statistics=True)
    assert np.array_equal(got, ref.get_populations(np.float32))
    assert ref.get_statistics() == st
    ref.close()


def test_lattice_allocation_failure_is_reported_and_the_next_one_succeeds():
    _fault(ALLOC, 1)
    with pytest.raises(lbx.LbxError) as e:
        lbx.BlockLattice(19, (16, 16, 16), (1, 1, 1), "f32")
    assert e.value.code == -5  # LBX_ERR_OUT_OF_MEMORY
    lat = lbx.BlockLattice(19, (16, 16, 16), (1, 1, 1), "f32")  # the one failure was used up
    lat.define_dynamics("bgk", omega=1.5)
    lat.collide_and_stream(2)
    lat.close()


def test_ensemble_allocation_failure_is_reported():
    _fault(ALLOC, 1)
    with pytest.raises(lbx.LbxError) as e:
        lbx.Ensemble(19, "f32", slab_bytes=64 << 20, max_lattices=4)
    assert e.value.code == -5
    with lbx.Ensemble(19, "f32", slab_bytes=64 << 20, max_lattices=4) as ens:
        assert ens.admit(lbx.make_request((16, 16, 16), 1.2, 0.05)) is not None


def test_cancelling_a_running_request_leaves_the_others_unchanged():
    """A request retired while running (cancelled) frees its slot; the other lattices continue
    exactly as they would have without it."""
    reqs = [lbx.make_request((24, 24, 24), 1.3, 0.05), lbx.make_request((16, 16, 16), 1.1, 0.05)]
    with lbx.Ensemble(19, "f32", slab_bytes=256 << 20, max_lattices=8) as a, \
            lbx.Ensemble(19, "f32", slab_bytes=256 << 20, max_lattices=8) as b:
        a0, a1 = a.admit(reqs[0]), a.admit(reqs[1])
        b1 = b.admit(reqs[1])
        a.run(30)
        b.run(30)
        a.retire(a0)  # cancelled mid-run
        assert a.admit(lbx.make_request((20, 20, 20), 1.2, 0.05)) is not None  # its memory is free again
        a.run(40)
        b.run(40)
        ra, ua = a.moments(a1)
        rb, ub = b.moments(b1)
        assert np.array_equal(ra, rb) and np.array_equal(ua, ub)
