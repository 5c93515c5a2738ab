"""Unit checks of the oracle itself (conversions, conservation) -- CPU only."""
import numpy as np
import pytest

import lbcases as L


def test_half_conversion_matches_numpy():
    lib = L.oracle()
    rng = np.random.default_rng(0)
    vals = np.concatenate([
        rng.normal(0, 1e-2, 4000), rng.normal(0, 1e-5, 2000), rng.normal(0, 100, 1000),
        np.array([0.0, -0.0, 65504.0, 65520.0, 1e-8, 6.0e-8, 2.0 ** -24, 2.0 ** -25, 2.0 ** -14, 1e5]),
    ]).astype(np.float32)
    for v in vals:
        want = np.array([v], np.float32).astype(np.float16).view(np.uint16)[0]
        got = lib.lbo_float_to_half(float(v))
        assert got == want, (v, hex(got), hex(want))
        assert np.float32(lib.lbo_half_to_float(got)) == np.float32(np.array([want], np.uint16).view(np.float16)[0])


def test_bf16_conversion_matches_torch():
    torch = pytest.importorskip("torch")
    lib = L.oracle()
    rng = np.random.default_rng(1)
    vals = np.concatenate([rng.normal(0, 1e-2, 3000), rng.normal(0, 1e3, 500)]).astype(np.float32)
    want = torch.from_numpy(vals).to(torch.bfloat16).view(torch.int16).numpy().view(np.uint16)
    for v, w in zip(vals, want):
        assert lib.lbo_float_to_bf16(float(v)) == w


@pytest.mark.parametrize("q", [9, 19, 27])
def test_oracle_conserves_mass_and_momentum_on_periodic_lattices(q):
    core = (6, 5, 1) if q == 9 else (5, 4, 6)
    rng = np.random.default_rng(q)
    n = int(np.prod(core))
    f = (rng.random((q, n)) - 0.5) * 0.02 * L.W[q][:, None]
    setup = {"q": q, "core": core, "periodic": (1, 1, 1 if q != 9 else 0), "dyn": "trt", "omega": 1.3,
             "magic": 0.25, "cs": 0.1, "force": [0, 0, 0], "links": None, "cell_dyn": None}
    out, _ = L.run_oracle(setup, f, 25)
    rho0, u0 = L.moments(q, f)
    rho1, u1 = L.moments(q, out)
    assert abs(rho1.sum() - rho0.sum()) < 1e-12 * n
    assert np.allclose((u1 * rho1).sum(axis=1), (u0 * rho0).sum(axis=1), atol=1e-13 * n)
