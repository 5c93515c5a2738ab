"""The CPU oracle against the reference's own CPU runs (golden fixtures).

FP64 fixtures come from the reference built with its DISABLE_CSE feature (generic dynamics
templates) and with the generated CSE kernels; FP32 fixtures from the float build.  The
oracle restates the generic templates, so it must agree with the FP64 runs to rounding
(<= 2e-12 of the largest population).  The CSE build of the Smagorinsky kernels carries
constants rounded to ~1e-7 (e.g. 3.00000046417339 for 3 in the D3Q19 kernel), which bounds
that comparison at 1e-7 instead.
"""
import numpy as np
import pytest

import lbcases as L

NAMES = L.fixture_names()


def _tolerances(name: str) -> tuple[float, float, float]:
    """(population, velocity L2, statistics) relative tolerances."""
    if name.endswith("_f32"):
        return 1e-4, 2e-5, 1e-5
    if name.endswith("_f64cse") and "smag" in name:
        return 1e-7, 1e-7, 1e-7
    return 2e-12, 1e-12, 1e-12


@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_reference(name):
    fx = L.load_fixture(name)
    meta = fx["meta"]
    setup = L.case_setup(fx)
    dt = np.float64 if meta["bytes"] == 8 else np.float32
    out, stats = L.run_oracle(setup, fx["f0"], meta["steps"], dtype=dt)
    forced = setup["force"] if setup["dyn"] in ("fbgk", "fsmag") else None
    e = L.errors(meta["q"], out, fx["fS"], L.fluid_mask(fx), forced)
    tp, tu, ts = _tolerances(name)
    assert e["pop"] <= tp, e
    assert e["u_l2"] <= tu, e
    ref = fx["stats"]
    every = meta.get("stats_every", 1)
    if every > 1:
        stats = np.vstack([stats[::every], stats[-1:]])
    rel = np.abs(stats - ref) / np.maximum(np.abs(ref), 1e-30)
    assert rel[:, 0].max() <= ts  # average rho
    assert rel[:, 2].max() <= max(ts, 1e-9)  # max |u|
    pops, cells = L.known_populations(fx) if len(L.local_flat_cells(fx)) else (None, None)
    if pops is not None:
        # the local flat cells: every population not entering from beyond the domain
        got, want = out[pops, cells], np.asarray(fx["fS"])[pops, cells]
        assert np.abs(got - want).max() <= tp * np.abs(fx["fS"]).max()


def test_fixture_set_covers_the_hot_path():
    have = set(NAMES)
    for q in ("d2q9", "d3q19", "d3q27"):
        for dyn in ("bgk", "trt", "smag", "fbgk", "fsmag"):
            for kind in ("f64", "f64cse", "f32"):
                assert f"periodic_{q}_{dyn}_{kind}" in have
    assert any(n.startswith("cavity_") and "_bb_" in n for n in have)
    assert any(n.startswith("cavity_") and "_bgk_" in n for n in have)
    assert any(n.startswith("porous_") for n in have)
