"""lbx_mass_momentum_noalloc: the mass/momentum sums for callers that cannot allocate device
memory (their device memory belongs to their own pool, or they run where the CUDA allocator
must not be entered).  The entry point keeps its scratch in a static device array instead of
calling cudaMalloc; here it is checked through the C ABI against the regular reduction
(lbx_reduce with LBX_REDUCE_MASS_MOMENTUM) of the same populations in every storage form, on two
calls in a row that each follow a call over a larger lattice, within the FP64 reduction
tolerance the other tests use (1e-12 relative).

This file is collected last on purpose: if it fails, a run that stops at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from openlb_b200 import lbx

pytestmark = pytest.mark.gpu

MAX_CELLS = 8192 * 4096


def _noalloc():
    fn = lbx.lib.lbx_mass_momentum_noalloc
    fn.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_int64, C.c_int64, C.POINTER(C.c_double), C.c_void_p]
    fn.restype = C.c_int
    return fn


def _lattice(q, core, storage, seed):
    rng = np.random.default_rng(seed)
    lat = lbx.BlockLattice(q, core, (1, 1, 1 if q != 9 else 0), storage)
    lat.define_dynamics("bgk", omega=1.4)
    n = int(np.prod(core))
    w = {9: 1 / 9, 19: 1 / 18, 27: 1 / 27}[q]
    lat.set_populations((rng.random((q, n)) - 0.5) * 0.02 * w)
    lat.collide_and_stream(10)
    return lat


def _device_populations(torch, lat, storage):
    """The lattice's populations (f - w) as a device array of its storage type, [q][cells]."""
    host = lat.get_populations(np.float64 if storage == "f64" else np.float32)
    dev = torch.from_numpy(host).to("cuda:0")
    if storage == "f16dev":
        dev = dev.to(torch.float16)  # exact: the values were stored in binary16
    elif storage == "bf16dev":
        dev = dev.to(torch.bfloat16)
    torch.cuda.synchronize()
    return dev.contiguous()


# tolerance relative to the mass: FP64 reductions of the same values in another order
TOL = 1e-12


@pytest.mark.parametrize("q,core,storage", [(19, (24, 20, 16), "f64"), (19, (64, 64, 64), "f32"),
                                            (27, (33, 17, 9), "f64"), (9, (300, 70, 1), "f32"),
                                            (19, (32, 32, 32), "f16dev"), (19, (32, 32, 32), "bf16dev")])
def test_noalloc_sums_match_regular_reduction(q, core, storage):
    torch = pytest.importorskip("torch")
    fn = _noalloc()
    # a large lattice first, then this one: the second call must not pick up partial sums the
    # first left in the shared scratch
    big = _lattice(19, (96, 96, 96), "f32", seed=99)
    big_dev = _device_populations(torch, big, "f32")
    lat = _lattice(q, core, storage, seed=q)
    want = lat.reduce(lbx.REDUCE_MASS_MOMENTUM)
    dev = _device_populations(torch, lat, storage)
    n = dev.shape[1]
    for _ in range(2):
        out = (C.c_double * 4)()
        rc = fn(19, lbx.STORAGE["f32"], C.c_void_p(big_dev.data_ptr()), big_dev.shape[1], big_dev.shape[1], out,
                None)
        assert rc == 0, lbx.lib.lbx_last_error().decode()
        out = (C.c_double * 4)()
        rc = fn(q, lbx.STORAGE[storage], C.c_void_p(dev.data_ptr()), n, n, out, None)
        assert rc == 0, lbx.lib.lbx_last_error().decode()
        got = np.array(out[:])
        assert abs(got[0] - want[0]) <= TOL * abs(want[0])
        assert np.allclose(got[1:], want[1:], rtol=0, atol=TOL * abs(want[0]))
    big.close()
    lat.close()


def test_noalloc_rejects_more_cells_than_the_scratch_holds():
    torch = pytest.importorskip("torch")
    dev = torch.zeros(19, dtype=torch.float32, device="cuda:0")
    out = (C.c_double * 4)()
    rc = _noalloc()(19, lbx.STORAGE["f32"], C.c_void_p(dev.data_ptr()), MAX_CELLS + 1, MAX_CELLS + 1, out, None)
    assert rc == -1
    assert "static scratch limit" in lbx.lib.lbx_last_error().decode()
