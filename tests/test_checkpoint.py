"""Checkpoint and resume (SuperLattice::save / load, core/serializer.h:77-79; the CUDA columns
serialise their data with the periodic-shift offset, core/platform/gpu/cuda/column.hh:305-321).

A run that is checkpointed, continued, and then resumed from the checkpoint in a fresh lattice
with the same set-up must reproduce the continued run bit for bit: populations and statistics.
The fresh lattice starts at shift 0 while the saved one had been rotated by the steps before
the checkpoint, so this also checks that the state does not depend on the shift.
"""
import numpy as np
import pytest

import lbcases as L
from openlb_b200 import lbx
from test_gpu_parity import make_lattice

pytestmark = pytest.mark.gpu

CASES = ["cavity_d3q19_bb_f64", "channel_d3q19_bgk_f64", "periodic_d3q19_trt_f64", "cavity_d2q9_bgk_f64"]


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("storage", ["f64", "f32", "f16dev", "bf16dev"])
def test_resume_reproduces_the_uninterrupted_run(name, storage):
    fx = L.load_fixture(name)
    setup = L.case_setup(fx)
    a = make_lattice(setup, storage)
    a.set_populations(np.asarray(fx["f0"], np.float64))
    a.post_process()
    a.collide_and_stream(23, statistics=True)
    ckpt = a.save_checkpoint()
    a.collide_and_stream(31, statistics=True)
    want, want_stats = a.get_populations(np.float64), a.get_statistics()
    a.close()

    b = make_lattice(setup, storage)
    b.load_checkpoint(ckpt)
    b.collide_and_stream(31, statistics=True)
    got, got_stats = b.get_populations(np.float64), b.get_statistics()
    b.close()
    assert np.array_equal(got, want)
    assert got_stats == want_stats


def test_checkpoint_carries_the_statistics():
    fx = L.load_fixture("cavity_d3q19_bgk_f64")
    setup = L.case_setup(fx)
    a = make_lattice(setup, "f64")
    a.set_populations(np.asarray(fx["f0"], np.float64))
    a.collide_and_stream(5, statistics=True)
    st = a.get_statistics()
    ckpt = a.save_checkpoint()
    a.close()
    b = make_lattice(setup, "f64")
    b.load_checkpoint(ckpt)
    assert b.get_statistics() == st
    b.close()


def test_checkpoint_of_another_lattice_is_refused():
    with lbx.BlockLattice(19, (12, 10, 8), (1, 1, 1), "f32") as a, \
            lbx.BlockLattice(19, (12, 10, 9), (1, 1, 1), "f32") as other, \
            lbx.BlockLattice(19, (12, 10, 8), (1, 1, 1), "f64") as wider, \
            lbx.BlockLattice(19, (12, 10, 8), (1, 1, 0), "f32") as walled:
        a.define_dynamics("bgk", omega=1.2)
        ckpt = a.save_checkpoint()
        for lat in (other, wider, walled):
            with pytest.raises(lbx.LbxError, match="checkpoint"):
                lat.load_checkpoint(ckpt)
        with pytest.raises(lbx.LbxError, match="checkpoint"):
            a.load_checkpoint(ckpt[:-8])  # truncated
        with pytest.raises(lbx.LbxError, match="checkpoint"):
            a.load_checkpoint(b"\0" * len(ckpt))  # not a checkpoint
        a.load_checkpoint(ckpt)  # its own checkpoint loads
