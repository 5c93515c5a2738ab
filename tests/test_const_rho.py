"""ConstRhoBGK (collision::ConstRhoBGK, dynamics/collision.h:322-351), the bulk dynamics of the
reference's cavity2d example.  Parity with the reference and the oracle runs through the
fixtures periodic_d2q9_constrho_*, periodic_d3q19_constrho_f64 and cavity_d2q9_constrho_f64 in
test_gpu_parity.py; these tests cover what the dynamics adds: the coupling to the previous
step's average density, in every storage form, across split calls, the autotuner and a
checkpoint.
"""
import numpy as np
import pytest

import lbcases as L
from openlb_b200 import lbx
from test_gpu_parity import make_lattice

pytestmark = pytest.mark.gpu


def _lattice(storage, fx):
    lat = make_lattice(L.case_setup(fx), storage)
    lat.set_populations(np.asarray(fx["f0"], np.float64))
    return lat


@pytest.mark.parametrize("storage,tol", [("f64", 1e-13), ("f32", 2e-6), ("f16dev", 2e-4), ("bf16dev", 2e-3)])
def test_average_density_is_pulled_back_to_one(storage, tol):
    """A random initial state averages 0.99892; after one step at AVERAGE_RHO = 1 the dynamics
    rescales every cell so the statistics' average returns to 1, as in the reference run."""
    fx = L.load_fixture("periodic_d2q9_constrho_f64")
    lat = _lattice(storage, fx)
    lat.collide_and_stream(1, statistics=True)
    first = lat.get_statistics()["average_rho"]
    lat.collide_and_stream(19, statistics=True)
    last = lat.get_statistics()["average_rho"]
    lat.close()
    assert abs(first - fx["stats"][0][0]) <= max(tol, 1e-12)
    assert abs(first - 1) > 1e-3  # the first step still runs at the initial average
    assert abs(last - 1) <= max(tol, 1e-15)


def test_statistics_are_kept_on_every_step():
    """The coupling needs the previous step's statistics even when the caller asks for none:
    steps run without statistics give the same bits as steps that ask for them."""
    fx = L.load_fixture("periodic_d3q19_constrho_f64")
    a, b = _lattice("f64", fx), _lattice("f64", fx)
    for _ in range(4):
        a.collide_and_stream(5, statistics=True)
    b.collide_and_stream(20)
    assert np.array_equal(a.get_populations(), b.get_populations())
    a.close()
    b.close()


def test_autotune_restores_the_statistics_it_steps_over():
    fx = L.load_fixture("periodic_d3q19_constrho_f64")
    lat = _lattice("f32", fx)
    lat.collide_and_stream(3, statistics=True)
    st = lat.get_statistics()
    before = lat.get_populations()
    lat.autotune(steps=3)
    assert lat.get_statistics() == st
    assert np.array_equal(lat.get_populations(), before)
    lat.close()


def test_resume_from_a_checkpoint_keeps_the_coupling():
    fx = L.load_fixture("cavity_d2q9_constrho_f64")
    a = _lattice("f64", fx)
    a.post_process()
    a.collide_and_stream(40)
    ckpt = a.save_checkpoint()
    a.collide_and_stream(30)
    want = a.get_populations()
    a.close()
    b = make_lattice(L.case_setup(fx), "f64")
    b.load_checkpoint(ckpt)
    b.collide_and_stream(30)
    assert np.array_equal(b.get_populations(), want)
    b.close()
