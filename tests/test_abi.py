"""The C ABI library without a GPU: it loads, exports every declared entry point, validates
arguments, refuses to run without a device, and its host-side link setter agrees with the
numpy restatement of setBouzidiBoundary."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import lbcases as L
from openlb_b200 import lbx

HEADERS = sorted((Path(__file__).resolve().parent.parent / "include").glob("*.h"))


def declared_functions() -> list[str]:
    text = "\n".join(h.read_text() for h in HEADERS)
    return sorted(set(re.findall(r"^(?:int|const char\*)\s+(lbx_\w+)\s*\(", text, flags=re.M)))


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) >= 18
    assert "lbx_server_create" in names and "lbx_mass_momentum_noalloc" in names
    lib = ctypes.CDLL(str(lbx.LIB_PATH))
    for n in names:
        assert hasattr(lib, n), n


def test_abi_version():
    assert lbx.lib.lbx_abi_version() == 1


def test_argument_validation_without_device():
    h = ctypes.c_void_p()
    core = (ctypes.c_int32 * 3)(4, 4, 4)
    per = (ctypes.c_int32 * 3)(0, 0, 0)
    assert lbx.lib.lbx_lattice_create(15, core, per, 1, 0, ctypes.byref(h)) == -4  # unsupported descriptor
    assert lbx.lib.lbx_lattice_create(19, core, per, 9, 0, ctypes.byref(h)) == -1  # unknown storage
    core2 = (ctypes.c_int32 * 3)(4, 4, 2)
    assert lbx.lib.lbx_lattice_create(9, core2, per, 1, 0, ctypes.byref(h)) == -1  # D2Q9 needs nz == 1
    assert lbx.lib.lbx_lattice_create(19, core, per, 1, 0, None) == -1


def test_no_silent_cpu_fallback():
    if lbx.device_count() > 0:
        pytest.skip("a GPU is visible")
    with pytest.raises(lbx.LbxError) as e:
        lbx.BlockLattice(19, (8, 8, 8))
    assert e.value.code == -2


@pytest.mark.parametrize("name", ["cavity_d2q9_bgk_f64", "cavity_d3q19_bgk_f64", "porous_d3q19_fbgk_f64",
                                  "porous_d2q9_trt_f64", "porous_d3q27_fsmag_f64"])
def test_link_setter_matches_restatement(name):
    fx = L.load_fixture(name)
    meta = fx["meta"]
    q, core, per = meta["q"], L.core_of(meta), L.periodic_of(meta)
    if meta["case"] == "cavity":
        solid, wv = (2, 3), [(0, 0, 0), (meta["ulid"], 0, 0)]
    else:
        solid, wv = (2,), None
    c1, d1, w1 = L.bouzidi_links(q, core, fx["mat"], 1, solid, wv, per)
    c2, d2, w2 = lbx.build_bouzidi_links(q, core, fx["mat"], 1, solid, wv, per)
    o2 = np.lexsort((d2, c2))
    assert np.array_equal(c1, c2[o2]) and np.array_equal(d1, d2[o2])
    assert np.allclose(w1, w2[o2], rtol=0, atol=0)
