"""Shared helpers of the test suite: golden fixtures, the CPU oracle binding, link derivation
and error metrics.  Test infrastructure only.

The oracle (oracle/lbm_oracle.c, built into oracle/_build/liblbmoracle.so) is the checker;
the CUDA path under test is openlb_b200.lbx.
"""
from __future__ import annotations

import ctypes as C
import json
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
ORACLE_LIB = ROOT / "oracle" / "_build" / "liblbmoracle.so"

# descriptor tables (src/descriptor/definition/common.h), used for moments and links
C9 = [(0, 0, 0), (-1, 1, 0), (-1, 0, 0), (-1, -1, 0), (0, -1, 0), (1, -1, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0)]
C19 = [(0, 0, 0), (-1, 0, 0), (0, -1, 0), (0, 0, -1), (-1, -1, 0), (-1, 1, 0), (-1, 0, -1), (-1, 0, 1),
       (0, -1, -1), (0, -1, 1), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (1, -1, 0), (1, 0, 1), (1, 0, -1),
       (0, 1, 1), (0, 1, -1)]
C27 = [(0, 0, 0), (-1, 0, 0), (0, -1, 0), (0, 0, -1), (-1, -1, 0), (-1, 1, 0), (-1, 0, -1), (-1, 0, 1),
       (0, -1, -1), (0, -1, 1), (-1, -1, -1), (-1, -1, 1), (-1, 1, -1), (-1, 1, 1), (1, 0, 0), (0, 1, 0),
       (0, 0, 1), (1, 1, 0), (1, -1, 0), (1, 0, 1), (1, 0, -1), (0, 1, 1), (0, 1, -1), (1, 1, 1), (1, 1, -1),
       (1, -1, 1), (1, -1, -1)]
VEL = {9: np.array(C9), 19: np.array(C19), 27: np.array(C27)}
W = {9: np.array([4 / 9] + [1 / 36, 1 / 9] * 4),
     19: np.array([1 / 3] + [1 / 18] * 3 + [1 / 36] * 6 + [1 / 18] * 3 + [1 / 36] * 6),
     27: np.array([8 / 27] + [2 / 27] * 3 + [1 / 54] * 6 + [1 / 216] * 4 + [2 / 27] * 3 + [1 / 54] * 6 + [1 / 216] * 4)}
DYN_CODE = {"bgk": 0, "trt": 1, "smag": 2, "fbgk": 3, "fsmag": 4, "constrho": 5}
GPU_DYN = {"bgk": "bgk", "trt": "trt", "smag": "smagorinsky_bgk", "fbgk": "forced_bgk",
           "fsmag": "smagorinsky_forced_bgk", "constrho": "const_rho_bgk"}


def opposite(q: int) -> np.ndarray:
    c = VEL[q]
    return np.array([int(np.where((c == -c[i]).all(axis=1))[0][0]) for i in range(q)])


# ---- fixtures -------------------------------------------------------------------------------
def fixture_names() -> list[str]:
    return sorted(p.stem for p in GOLDEN.glob("*.npz"))


def load_fixture(name: str) -> dict:
    z = np.load(GOLDEN / f"{name}.npz")
    meta = json.loads(str(z["meta"]))
    fx = {k: z[k] for k in ("f0", "fS", "mat", "stats")}
    for k in ("bnd", "vals", "bclass", "force"):
        if k in z.files:
            fx[k] = z[k]
    fx["meta"] = meta
    fx["name"] = name
    return fx


def core_of(meta: dict) -> tuple[int, int, int]:
    e = meta["ext"]
    return int(e[0]), int(e[1]), int(e[2])


def periodic_of(meta: dict) -> tuple[int, int, int]:
    if meta["case"] == "geo":
        return tuple(int(v) for v in meta["periodic"])
    if meta["case"] == "channel":  # inlet/outlet along x, periodic across
        return (0, 1, 1 if meta["d"] == 3 else 0)
    p = 1 if meta["case"] in ("periodic", "porous") else 0
    return (p, p, p if meta["d"] == 3 else 0)


# ---- halfway bounce-back links: numpy restatement of setBouzidiBoundary's q = 1/2 fallback ----
def bouzidi_links(q: int, core, material: np.ndarray, fluid: int, solid, wall_velocity=None, periodic=(0, 0, 0)):
    """Links (x_b, k) with x_b fluid and x_b + c_k solid (boundary/setBouzidiBoundary.h:236-330);
    wall term c_k . u_wall of the solid material (setBouzidiVelocity, :386-410)."""
    nx, ny, nz = core
    mat = material.reshape(nx, ny, nz)
    c = VEL[q]
    cells, dirs, wall = [], [], []
    idx = np.arange(nx * ny * nz).reshape(nx, ny, nz)
    X, Y, Z = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    fl = mat == fluid
    for k in range(1, q):
        sx, sy, sz = X + c[k][0], Y + c[k][1], Z + c[k][2]
        ok = np.ones_like(fl)
        for s, n, per in ((sx, nx, periodic[0]), (sy, ny, periodic[1]), (sz, nz, periodic[2])):
            if per:
                s %= n
            else:
                ok &= (s >= 0) & (s < n)
        sxc, syc, szc = np.clip(sx, 0, nx - 1), np.clip(sy, 0, ny - 1), np.clip(sz, 0, nz - 1)
        smat = mat[sxc, syc, szc]
        for j, m in enumerate(solid):
            hit = fl & ok & (smat == m)
            n_hit = int(hit.sum())
            if n_hit:
                cells.append(idx[hit])
                dirs.append(np.full(n_hit, k))
                uw = np.zeros(3) if wall_velocity is None else np.asarray(wall_velocity[j], float)
                wall.append(np.full(n_hit, float(np.dot(c[k], uw))))
    if not cells:
        return np.zeros(0, np.int64), np.zeros(0, np.int32), np.zeros(0)
    cells = np.concatenate(cells)
    dirs = np.concatenate(dirs).astype(np.int32)
    wall = np.concatenate(wall)
    order = np.lexsort((dirs, cells))
    return cells[order].astype(np.int64), dirs[order], wall[order]


def case_setup(fx: dict) -> dict:
    """Dynamics, per-cell map and links of a fixture, as the reference driver set them up."""
    meta = fx["meta"]
    q = meta["q"]
    core = core_of(meta)
    per = periodic_of(meta)
    mat = fx["mat"]
    setup = {"q": q, "core": core, "periodic": per, "dyn": meta["dyn"], "omega": meta["omega"],
             "magic": meta["magic"], "cs": meta["cs"], "force": list(meta["force"]), "links": None,
             "cell_dyn": None, "fd": None}
    if meta["case"] == "cavity":
        if meta["walls"] == "bounceback":
            cd = np.where(mat == 1, 1, 2).astype(np.uint8)
        else:
            cd = np.where(mat == 1, 1, 0).astype(np.uint8)
            setup["links"] = bouzidi_links(q, core, mat, 1, (2, 3), [(0, 0, 0), (meta["ulid"], 0, 0)], per)
        setup["cell_dyn"] = cd
    elif meta["case"] == "porous":
        if meta["walls"] == "bounceback":
            setup["cell_dyn"] = np.where(mat == 1, 1, 2).astype(np.uint8)
        else:
            setup["cell_dyn"] = np.where(mat == 1, 1, 0).astype(np.uint8)
            setup["links"] = bouzidi_links(q, core, mat, 1, (2,), None, per)
    elif meta["case"] == "geo":
        a = geo_args(meta)
        mat3 = mat.reshape(core)
        cd = np.zeros(mat.shape, np.uint8)
        cd[mat == 1] = 1
        for m in a["bounceback"]:
            cd[mat == m] = 2
        solid = list(a["bouzidi"])
        walls = [(0.0, 0.0, 0.0)] * len(solid)
        if a["lid"] is not None:
            solid.append(a["lid"])
            walls.append((meta["ulid"], 0.0, 0.0))
        if solid:
            setup["links"] = bouzidi_links(q, core, mat3, 1, solid, walls if a["lid"] is not None else None, per)
        for m in a["bbvel"]:
            cd[mat == m] = 4
        if a["bgk_mat"] is not None:
            # the second fluid dynamics, parameter class 1 (cell id 8): BGK beside ForcedBGK is the
            # forced dynamics with a zero force; beside another kind it is BGK itself
            cd[mat == a["bgk_mat"]] = 8
            setup["classes"] = {1: {"omega": meta["omega"], "magic": meta["magic"], "cs": meta["cs"],
                                    "force": [0.0, 0.0, 0.0],
                                    "dyn": None if meta["dyn"] in ("bgk", "fbgk") else "bgk"}}
        if a["trt_mat"] is not None:
            cd[mat == a["trt_mat"]] = 8
            setup["classes"] = {1: {"omega": meta["omega"], "magic": meta["magic"], "cs": meta["cs"],
                                    "force": [0.0, 0.0, 0.0], "dyn": None if meta["dyn"] == "trt" else "trt"}}
        if a["bbvel"]:
            cells = np.nonzero(np.isin(mat, a["bbvel"]))[0].astype(np.int64)
            setup["bbv"] = {"cells": cells, "rho": np.ascontiguousarray(fx["vals"][cells, 0]),
                            "u": np.ascontiguousarray(fx["vals"][cells, 1:4])}
        bc = fx["bclass"] if "bclass" in fx else np.zeros((0, 6), np.int32)
        cd[bc[:, 0]] = 3
        setup["cell_dyn"] = cd
        kinds = bc[:, 1].astype(np.int32)
        if a["local"]:
            # LocalVelocity / LocalPressure: kinds 3 and 4 (BGK mixin), 5 and 6 (RLB mixin)
            kinds = kinds + (4 if a["rlb"] else 2)
        setup["fd"] = {"cells": bc[:, 0].astype(np.int64), "kinds": kinds,
                       "types": bc[:, 2].astype(np.int32), "normals": np.ascontiguousarray(bc[:, 3:6], np.int32),
                       "values": np.ascontiguousarray(fx["vals"][bc[:, 0]])}
    elif meta["case"] == "channel":
        # bulk dynamics on 1, bounce-back on the layers behind the open faces (2), BGK with
        # the boundary momenta on the inlet (3) and outlet (4) faces
        setup["cell_dyn"] = np.select([mat == 1, mat == 2], [1, 2], 3).astype(np.uint8)
        setup["fd"] = fd_boundaries(fx["bnd"])
    return setup


def geo_args(meta: dict) -> dict:
    """The boundary set-up of a "geo" fixture, read back from the driver arguments it was made
    with (oracle/ref_driver.cpp, geo case)."""
    args = meta["args"]

    def value(flag):
        return args[args.index(flag) + 1] if flag in args else None

    def ints(flag):
        v = value(flag)
        return [int(x) for x in v.split(",")] if v else []

    lid = value("--lid")
    return {"bouzidi": ints("--bouzidi"), "bounceback": ints("--bounceback"), "ivel": ints("--ivel"),
            "ivel_lid": ints("--ivel-lid"), "ipres": ints("--ipres"), "lid": int(lid) if lid else None,
            "bbvel": ints("--bbvel"), "local": "--local" in args or "--local-rlb" in args,
            "rlb": "--local-rlb" in args,
            "bgk_mat": int(value("--bgk-mat")) if value("--bgk-mat") else None,
            "trt_mat": int(value("--trt-mat")) if value("--trt-mat") else None,
            "force_mat": ints("--force-mat")}


def fd_boundaries(bnd: np.ndarray) -> dict:
    """Flat-face boundary list of the reference driver's channel case (rows of
    {cell, kind, direction, orientation, value[4]})."""
    b = np.asarray(bnd, np.float64).reshape(-1, 8)
    return {"cells": b[:, 0].astype(np.int64), "kinds": b[:, 1].astype(np.int32),
            "dirs": b[:, 2].astype(np.int32), "orients": b[:, 3].astype(np.int32),
            "values": np.ascontiguousarray(b[:, 4:8])}


# ---- oracle -----------------------------------------------------------------------------------
class _Case(C.Structure):
    _fields_ = [("q", C.c_int32), ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("periodic", C.c_int32), ("dynamics", C.c_int32), ("omega", C.c_double), ("magic", C.c_double),
                ("smagorinsky", C.c_double), ("force", C.c_double * 3), ("material", C.c_void_p),
                ("n_links", C.c_int64), ("link_cell", C.c_void_p), ("link_dir", C.c_void_p),
                ("link_wall", C.c_void_p), ("n_fd", C.c_int64), ("fd_cell", C.c_void_p),
                ("fd_kind", C.c_void_p), ("fd_dir", C.c_void_p), ("fd_orient", C.c_void_p),
                ("fd_value", C.c_void_p), ("fd_type", C.c_void_p), ("fd_normal", C.c_void_p),
                ("bbv_value", C.c_void_p), ("class_params", C.c_void_p), ("class_dynamics", C.c_void_p)]


_oracle = None


def oracle():
    global _oracle
    if _oracle is None:
        if not ORACLE_LIB.exists():
            subprocess.run(["make", "-C", str(ROOT / "oracle"), "oracle"], check=True, capture_output=True)
        lib = C.CDLL(str(ORACLE_LIB))
        for fn in ("lbo_run_f64", "lbo_run_f32"):
            getattr(lib, fn).argtypes = [C.POINTER(_Case), C.c_void_p, C.c_int64, C.c_void_p]
            getattr(lib, fn).restype = C.c_int
        lib.lbo_run_half.argtypes = [C.POINTER(_Case), C.c_void_p, C.c_int32, C.c_int64, C.c_void_p]
        lib.lbo_run_half.restype = C.c_int
        lib.lbo_float_to_half.argtypes = [C.c_float]
        lib.lbo_float_to_half.restype = C.c_uint16
        lib.lbo_half_to_float.argtypes = [C.c_uint16]
        lib.lbo_half_to_float.restype = C.c_float
        lib.lbo_float_to_bf16.argtypes = [C.c_float]
        lib.lbo_float_to_bf16.restype = C.c_uint16
        lib.lbo_bf16_to_float.argtypes = [C.c_uint16]
        lib.lbo_bf16_to_float.restype = C.c_float
        _oracle = lib
    return _oracle


def run_oracle(setup: dict, f: np.ndarray, steps: int, dtype=np.float64, storage: str | None = None):
    """Run the oracle in place on a copy of f; returns (f, stats[steps, 3])."""
    lib = oracle()
    keep = []
    c = _Case()
    c.q = setup["q"]
    c.nx, c.ny, c.nz = setup["core"]
    per = setup["periodic"]
    c.periodic = (1 if per[0] else 0) | (2 if per[1] else 0) | (4 if len(per) > 2 and per[2] else 0)
    c.dynamics = DYN_CODE[setup["dyn"]]
    c.omega, c.magic, c.smagorinsky = setup["omega"], setup["magic"], setup["cs"]
    c.force = (C.c_double * 3)(*(list(setup["force"]) + [0.0] * 3)[:3])
    if setup["cell_dyn"] is not None:
        cd = setup["cell_dyn"]
        m = np.select([cd == 1, cd == 2, cd == 3, cd == 4, cd == 8, cd == 9, cd == 10], [1, 4, 5, 6, 8, 9, 10],
                      0).astype(np.int32)
        keep.append(m)
        c.material = m.ctypes.data
    if setup.get("fd") is not None:
        fd = setup["fd"]
        if "normals" in fd:
            arrs = [np.ascontiguousarray(fd[k]) for k in ("cells", "kinds", "values", "types", "normals")]
            keep += arrs
            c.n_fd = len(arrs[0])
            c.fd_cell, c.fd_kind, c.fd_value, c.fd_type, c.fd_normal = (a.ctypes.data for a in arrs)
        else:
            arrs = [np.ascontiguousarray(fd[k]) for k in ("cells", "kinds", "dirs", "orients", "values")]
            keep += arrs
            c.n_fd = len(arrs[0])
            c.fd_cell, c.fd_kind, c.fd_dir, c.fd_orient, c.fd_value = (a.ctypes.data for a in arrs)
    if setup.get("bbv") is not None:
        n_all = int(np.prod(setup["core"]))
        bv = np.zeros((n_all, 4))
        b = setup["bbv"]
        bv[b["cells"], 0] = b["rho"]
        bv[b["cells"], 1:4] = b["u"]
        keep.append(bv)
        c.bbv_value = bv.ctypes.data
    if setup.get("classes"):
        cp = np.zeros((3, 6))
        cdyn = np.full(3, -1, np.int32)
        for k, prm in setup["classes"].items():
            cp[k - 1] = [prm["omega"], prm["magic"], prm["cs"], *list(prm["force"])[:3]]
            if prm.get("dyn"):
                cdyn[k - 1] = DYN_CODE[prm["dyn"]]
        keep += [cp, cdyn]
        c.class_params = cp.ctypes.data
        c.class_dynamics = cdyn.ctypes.data
    if setup["links"] is not None:
        cells, dirs, wall = (np.ascontiguousarray(a) for a in setup["links"])
        keep += [cells, dirs, wall]
        c.n_links = len(cells)
        c.link_cell, c.link_dir, c.link_wall = cells.ctypes.data, dirs.ctypes.data, wall.ctypes.data
    stats = np.zeros((max(steps, 1), 3))
    if storage in ("f16dev", "bf16dev"):
        conv = lib.lbo_float_to_half if storage == "f16dev" else lib.lbo_float_to_bf16
        flat = np.ascontiguousarray(f, dtype=np.float32).reshape(-1)
        h = np.array([conv(float(v)) for v in flat], dtype=np.uint16)
        rc = lib.lbo_run_half(C.byref(c), h.ctypes.data, 1 if storage == "f16dev" else 2, steps, stats.ctypes.data)
        back = lib.lbo_half_to_float if storage == "f16dev" else lib.lbo_bf16_to_float
        out = np.array([back(int(v)) for v in h], dtype=np.float32).reshape(f.shape)
    else:
        out = np.ascontiguousarray(f, dtype=dtype).copy()
        fn = lib.lbo_run_f64 if dtype == np.float64 else lib.lbo_run_f32
        rc = fn(C.byref(c), out.ctypes.data, steps, stats.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"oracle failed: {rc}")
    return out, stats[:steps]


# ---- metrics ------------------------------------------------------------------------------------
def moments(q: int, f: np.ndarray, force=None):
    f = np.asarray(f, np.float64)
    c = VEL[q][:, : (2 if q == 9 else 3)]
    rho = f.sum(axis=0) + 1.0
    u = (c.T @ f) / rho
    if force is not None:
        u = u + 0.5 * np.asarray(force[: u.shape[0]])[:, None]
    return rho, u


def errors(q: int, a: np.ndarray, b: np.ndarray, mask: np.ndarray | None = None, force=None) -> dict:
    """Relative errors of a against b over the cells in mask: populations (max abs diff over
    max |b|), velocity (max and L2) and density (max abs)."""
    if mask is not None:
        a, b = a[:, mask], b[:, mask]
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    ra, ua = moments(q, a, force)
    rb, ub = moments(q, b, force)
    umax = np.abs(ub).max() or 1.0
    return {
        "pop": float(np.abs(a - b).max() / (np.abs(b).max() or 1.0)),
        "u_inf": float(np.abs(ua - ub).max() / umax),
        "u_l2": float(np.sqrt(((ua - ub) ** 2).sum() / max((ub ** 2).sum(), 1e-300))),
        "rho_inf": float(np.abs(ra - rb).max()),
    }


def fluid_mask(fx: dict) -> np.ndarray:
    """Cells whose populations are compared: the bulk fluid, and in the channel also the
    inlet and outlet faces (materials 3 and 4; in the cavity those numbers are walls)."""
    if fx["meta"]["case"] == "channel":
        return np.isin(fx["mat"], (1, 3, 4))
    if fx["meta"]["case"] == "geo":
        m = fx["mat"] == 1
        for second in (geo_args(fx["meta"])["bgk_mat"], geo_args(fx["meta"])["trt_mat"]):
            if second is not None:
                m |= fx["mat"] == second
        if "bclass" in fx:
            m[fx["bclass"][:, 0]] = True
        m[local_flat_cells(fx)] = False
        return m
    return fx["mat"] == 1


def local_flat_cells(fx: dict) -> np.ndarray:
    """Cells regularised in their collision whose populations entering from beyond the domain
    are, after a stream, whatever the cells there held (in the reference: its storage's
    leftovers): the flat cells of a LocalVelocity / LocalPressure boundary and the internal
    edges and corners of any velocity boundary.  The next collision rebuilds those populations
    from the others, so only the others are compared (known_populations)."""
    if fx["meta"]["case"] != "geo" or "bclass" not in fx:
        return np.zeros(0, np.int64)
    bc = fx["bclass"]
    pick = np.isin(bc[:, 2], (2, 4))
    if geo_args(fx["meta"])["local"]:
        pick |= bc[:, 2] == 0
    return bc[pick, 0].astype(np.int64)


def _unknown(vel: np.ndarray, i: int, ntype: int, n: np.ndarray) -> bool:
    """Population i enters from beyond the domain: c_i . n < 0 on a flat cell; c_i = -n along
    every normal axis of an internal corner, and along the two normal axes of an internal edge."""
    c = vel[i, :3]
    if ntype == 0:
        return int(np.dot(c, n)) < 0
    axes = [a for a in range(3) if n[a] != 0]
    return all(c[a] == -n[a] for a in axes)


def known_populations(fx: dict) -> tuple[np.ndarray, np.ndarray]:
    """(population, cell) index pairs of the cells of local_flat_cells whose populations do not
    enter from beyond the domain."""
    bc = fx["bclass"]
    q = fx["meta"]["q"]
    vel = VEL[q]
    cells_of = set(local_flat_cells(fx).tolist())
    pops, cells = [], []
    for row in bc:
        if int(row[0]) not in cells_of:
            continue
        n = row[3:6]
        for i in range(q):
            if not _unknown(vel, i, int(row[2]), n):
                pops.append(i)
                cells.append(int(row[0]))
    return np.asarray(pops, np.int64), np.asarray(cells, np.int64)


def counted_cells(fx: dict) -> int:
    """Cells the lattice statistics count: the compared cells, plus the bounce-back cells with a
    wall velocity (their populations arriving from beyond the domain are not defined, so they are
    not compared, but they report {rho, |u|^2})."""
    n = int(fluid_mask(fx).sum())
    if fx["meta"]["case"] == "geo":
        n += int(np.isin(fx["mat"], geo_args(fx["meta"])["bbvel"]).sum())
        n += len(local_flat_cells(fx))
    return n
