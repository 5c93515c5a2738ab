"""ctypes binding of liblbx.so (include/lbx.h) and a block-lattice wrapper.

`BlockLattice` mirrors the part of the reference's BlockLattice / SuperLattice interface
that drives the hot path (OpenLB 1.8r1, paths relative to the reference project):

    defineDynamics / setParameter   core/blockLattice.h:559-576  -> define_dynamics / set_parameter
    iniEquilibrium                  core/blockLattice.hh:201-219 -> ini_equilibrium
    collideAndStream                core/superLattice.hh:664-725 -> collide_and_stream
    getStatistics                   core/latticeStatistics.h:91-93 -> get_statistics
    setBouzidiBoundary/-Velocity    boundary/setBouzidiBoundary.h:193-420 -> set_bouzidi_boundary
    setProcessingContext(Evaluation) + cell access                  -> get_populations / compute_moments

There is no CPU fallback: importing this module fails when liblbx.so is missing, and
creating a lattice fails without an sm_100 GPU.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(os.environ.get("LBX_LIBRARY", Path(__file__).resolve().parent / "lib" / "liblbx.so"))

LBX_OK = 0
STORAGE = {"f64": 0, "f32": 1, "f16dev": 2, "bf16dev": 3}
STORAGE_BYTES = {"f64": 8, "f32": 4, "f16dev": 2, "bf16dev": 2}
DYNAMICS = {"bgk": 1, "trt": 2, "smagorinsky_bgk": 3, "forced_bgk": 4, "smagorinsky_forced_bgk": 5,
            "const_rho_bgk": 6}
CELL_NONE, CELL_BULK, CELL_BOUNCE_BACK, CELL_FD_BOUNDARY, CELL_BOUNCE_BACK_VELOCITY = 0, 1, 2, 3, 4
CELL_BULK_CLASS_1, CELL_BULK_CLASS_2, CELL_BULK_CLASS_3 = 8, 9, 10
STEP_STATISTICS = 1
REDUCE_MASS_MOMENTUM, REDUCE_DRAG, REDUCE_RESIDUAL = 1, 2, 3


class Params(C.Structure):
    _fields_ = [("omega", C.c_double), ("magic", C.c_double), ("smagorinsky", C.c_double),
                ("force", C.c_double * 3)]


class Info(C.Structure):
    _fields_ = [("q", C.c_int32), ("d", C.c_int32), ("core", C.c_int32 * 3), ("padded", C.c_int32 * 3),
                ("pad", C.c_int32), ("periodic", C.c_int32 * 3), ("storage", C.c_int32),
                ("n_cells", C.c_int64), ("n_core", C.c_int64), ("column_stride", C.c_int64),
                ("bytes", C.c_int64), ("n_links", C.c_int64), ("column_period", C.c_int64)]


class EnsembleRequest(C.Structure):
    _fields_ = [("core", C.c_int32 * 3), ("dynamics", C.c_int32), ("params", Params), ("lid_velocity", C.c_double),
                ("tolerance", C.c_double), ("max_steps", C.c_int64)]


class EnsembleStatus(C.Structure):
    _fields_ = [("state", C.c_int32), ("pad", C.c_int32), ("steps", C.c_int64), ("residual", C.c_double)]


class TuneEntry(C.Structure):
    _fields_ = [("variant", C.c_int32), ("block_x", C.c_int32), ("block_y", C.c_int32),
                ("cells_per_thread", C.c_int32), ("threads", C.c_int32), ("blocks_per_sm", C.c_int32),
                ("ms_per_step", C.c_double)]


def _tune(fn, handle, steps: int, stream, where: str) -> list[dict]:
    cap = 128
    arr = (TuneEntry * cap)()
    n = C.c_int32()
    check(fn(handle, steps, arr, cap, C.byref(n), _stream_ptr(stream)), where)
    return [{k: getattr(arr[i], k) for k, _ in TuneEntry._fields_} for i in range(min(n.value, cap))]


SLOT_FREE, SLOT_RUNNING, SLOT_CONVERGED, SLOT_MAX_STEPS, SLOT_DIVERGED = 0, 1, 2, 3, 4
SERVER_REJECTED, SERVER_CANCELLED = 5, 6


class ServerRequest(C.Structure):
    _fields_ = [("id", C.c_int64), ("arrival", C.c_double), ("request", EnsembleRequest)]


class ServerRecord(C.Structure):
    _fields_ = [("id", C.c_int64), ("cells", C.c_int64), ("arrival", C.c_double), ("admitted", C.c_double),
                ("finished", C.c_double), ("steps", C.c_int64), ("state", C.c_int32), ("slot", C.c_int32),
                ("residual", C.c_double)]


class ServerConfig(C.Structure):
    _fields_ = [("min_chunk", C.c_int32), ("max_chunk", C.c_int32), ("realtime", C.c_int32), ("pad", C.c_int32)]


ENGINE_ADMIT = C.CFUNCTYPE(C.c_int32, C.c_void_p, C.POINTER(EnsembleRequest), C.POINTER(C.c_int32))
ENGINE_RUN = C.CFUNCTYPE(C.c_int32, C.c_void_p, C.c_int32)
ENGINE_STATUSES = C.CFUNCTYPE(C.c_int32, C.c_void_p, C.POINTER(EnsembleStatus), C.c_int32)
ENGINE_RETIRE = C.CFUNCTYPE(C.c_int32, C.c_void_p, C.c_int32)
FINISH_FN = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(ServerRecord))


class ServerEngine(C.Structure):
    _fields_ = [("admit", ENGINE_ADMIT), ("run", ENGINE_RUN), ("statuses", ENGINE_STATUSES),
                ("retire", ENGINE_RETIRE), ("slots", C.c_int32), ("pad", C.c_int32)]


class ServerStats(C.Structure):
    _fields_ = [(k, C.c_int64) for k in ("submitted", "pending", "waiting", "running", "finished", "runs", "steps",
                                         "short_runs", "long_runs")] + [("busy_seconds", C.c_double),
                                                                         ("clock", C.c_double)]


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(f"liblbx.so not built ({LIB_PATH}); run `python -m openlb_b200.build`")
    lib = C.CDLL(str(LIB_PATH))
    P, I32, I64, U32, D, VP = C.POINTER, C.c_int32, C.c_int64, C.c_uint32, C.c_double, C.c_void_p
    sig = {
        "lbx_last_error": ([], C.c_char_p),
        "lbx_abi_version": ([], C.c_int),
        "lbx_device_count": ([], C.c_int),
        "lbx_lattice_create": ([I32, P(I32), P(I32), I32, I32, P(VP)], C.c_int),
        "lbx_lattice_destroy": ([VP], C.c_int),
        "lbx_get_info": ([VP, P(Info)], C.c_int),
        "lbx_set_dynamics": ([VP, I32, P(Params)], C.c_int),
        "lbx_set_cell_dynamics": ([VP, VP], C.c_int),
        "lbx_set_dynamics_class": ([VP, I32, P(Params)], C.c_int),
        "lbx_set_dynamics_class_kind": ([VP, I32, I32, P(Params)], C.c_int),
        "lbx_set_bouzidi_links": ([VP, I64, VP, VP, VP], C.c_int),
        "lbx_set_bouzidi_from_materials": ([VP, VP, I32, I32, VP, VP], C.c_int),
        "lbx_build_bouzidi_links": ([I32, P(I32), P(I32), VP, I32, I32, VP, VP, I64, VP, VP, VP, P(I64)], C.c_int),
        "lbx_upload_populations": ([VP, VP, I32, VP], C.c_int),
        "lbx_download_populations": ([VP, VP, I32, VP], C.c_int),
        "lbx_checkpoint_bytes": ([VP, P(I64)], C.c_int),
        "lbx_save_checkpoint": ([VP, VP, I64, VP], C.c_int),
        "lbx_load_checkpoint": ([VP, VP, I64, VP], C.c_int),
        "lbx_ini_equilibrium": ([VP, VP, VP, VP], C.c_int),
        "lbx_collide_and_stream": ([VP, I64, U32, VP], C.c_int),
        "lbx_get_statistics": ([VP, P(D), VP], C.c_int),
        "lbx_compute_moments": ([VP, VP, VP, VP], C.c_int),
        "lbx_reduce": ([VP, I32, P(D), VP], C.c_int),
        "lbx_boundary_force": ([VP, I32, P(D), VP], C.c_int),
        "lbx_population_shift": ([VP, I32, P(I64)], C.c_int),
        "lbx_rotate": ([VP, I32, I64], C.c_int),
        "lbx_population_ptr": ([VP, I32, P(VP), P(I64)], C.c_int),
        "lbx_set_launch_config": ([VP, I32, I32, I32, I32], C.c_int),
        "lbx_set_kernel_timing": ([VP, I32], C.c_int),
        "lbx_post_process": ([VP, VP], C.c_int),
        "lbx_set_fd_boundaries": ([VP, I64, VP, VP, VP, VP, VP], C.c_int),
        "lbx_set_boundary_cells": ([VP, I64, VP, VP, VP, VP, VP], C.c_int),
        "lbx_set_bounce_back_velocity": ([VP, I64, VP, VP, VP], C.c_int),
        "lbx_set_interpolated_boundary": ([VP, I32, VP, I32, I32, VP, I32, VP, VP], C.c_int),
        "lbx_discrete_normals": ([I32, P(I32), P(I32), VP, I32, I32, VP, I32, VP, I64, VP, VP, VP, P(I64)],
                                 C.c_int),
        "lbx_autotune": ([VP, I32, VP, I32, P(I32), VP], C.c_int),
        "lbx_ensemble_autotune": ([VP, I32, VP, I32, P(I32), VP], C.c_int),
        "lbx_ensemble_set_launch_mode": ([VP, I32], C.c_int),
        "lbx_ensemble_set_cells_per_thread": ([VP, I32], C.c_int),
        "lbx_ensemble_checkpoint_bytes": ([VP, I32, P(I64)], C.c_int),
        "lbx_ensemble_save_slot": ([VP, I32, VP, I64, VP], C.c_int),
        "lbx_ensemble_restore_slot": ([VP, VP, I64, P(I32), VP], C.c_int),
        "lbx_ensemble_footprint": ([I32, I32, P(EnsembleRequest), P(I64)], C.c_int),
        "lbx_ensemble_create": ([I32, I32, I64, I32, I32, P(VP)], C.c_int),
        "lbx_ensemble_destroy": ([VP], C.c_int),
        "lbx_ensemble_admit": ([VP, P(EnsembleRequest), P(I32)], C.c_int),
        "lbx_ensemble_run": ([VP, I32, VP], C.c_int),
        "lbx_ensemble_statuses": ([VP, P(EnsembleStatus), I32, VP], C.c_int),
        "lbx_ensemble_moments": ([VP, I32, VP, VP, VP], C.c_int),
        "lbx_ensemble_retire": ([VP, I32], C.c_int),
        "lbx_ensemble_set_config": ([VP, I32, I32, I32], C.c_int),
        "lbx_get_kernel_timing": ([VP, P(D)], C.c_int),
        "lbx_slabs_create": ([I32, P(I32), P(I32), I32, I32, VP, P(VP)], C.c_int),
        "lbx_slabs_destroy": ([VP], C.c_int),
        "lbx_slabs_get": ([VP, I32, P(VP), P(I32), P(I32)], C.c_int),
        "lbx_slabs_collide_and_stream": ([VP, I64, U32], C.c_int),
        "lbx_slabs_synchronize": ([VP], C.c_int),
        "lbx_slabs_get_statistics": ([VP, P(D)], C.c_int),
        "lbx_server_create": ([VP, I32, P(ServerConfig), VP, P(VP)], C.c_int),
        "lbx_server_create_with_engine": ([P(ServerEngine), VP, P(ServerConfig), P(VP)], C.c_int),
        "lbx_server_set_finish_callback": ([VP, FINISH_FN, VP], C.c_int),
        "lbx_server_submit": ([VP, P(ServerRequest), I32], C.c_int),
        "lbx_server_start": ([VP], C.c_int),
        "lbx_server_close": ([VP], C.c_int),
        "lbx_server_cancel": ([VP, I64], C.c_int),
        "lbx_server_wait": ([VP, D, P(I32)], C.c_int),
        "lbx_server_records": ([VP, P(ServerRecord), I32, P(I32)], C.c_int),
        "lbx_server_get_stats": ([VP, P(ServerStats)], C.c_int),
        "lbx_server_destroy": ([VP], C.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return lib


lib = _load()


class LbxError(RuntimeError):
    """A liblbx call failed (the C++ platform layer raises std::runtime_error likewise)."""

    def __init__(self, code: int, where: str):
        msg = lib.lbx_last_error().decode(errors="replace")
        super().__init__(f"{where} failed ({code}): {msg}")
        self.code = code


def check(code: int, where: str) -> None:
    if code != LBX_OK:
        raise LbxError(code, where)


def _ptr(a: np.ndarray | None) -> C.c_void_p | None:
    return None if a is None else C.c_void_p(a.ctypes.data)


def _i32x3(v) -> C.Array:
    return (C.c_int32 * 3)(*[int(x) for x in v])


def _stream_ptr(stream) -> C.c_void_p | None:
    if stream is None:
        return None
    if isinstance(stream, int):
        return C.c_void_p(stream)
    return C.c_void_p(int(stream.cuda_stream))  # torch.cuda.Stream


def device_count() -> int:
    return int(lib.lbx_device_count())


def build_bouzidi_links(q: int, core, material: np.ndarray, fluid: int = 1, solid=(2,),
                        wall_velocity=None, periodic=(False, False, False)):
    """Halfway bounce-back links of a material map, as setBouzidiBoundary derives them
    (q = 1/2 fallback).  Returns (cells int64, dirs int32, wall int32) numpy arrays."""
    mat = np.ascontiguousarray(material, dtype=np.int32).reshape(-1)
    sol = np.ascontiguousarray(solid, dtype=np.int32)
    wv = None if wall_velocity is None else np.ascontiguousarray(wall_velocity, dtype=np.float64).reshape(-1)
    n = C.c_int64(0)
    args = (q, _i32x3(core), _i32x3(periodic), _ptr(mat), fluid, len(sol), _ptr(sol), _ptr(wv))
    check(lib.lbx_build_bouzidi_links(*args, 0, None, None, None, C.byref(n)), "lbx_build_bouzidi_links")
    cells = np.zeros(n.value, np.int64)
    dirs = np.zeros(n.value, np.int32)
    wall = np.zeros(n.value, np.float64)
    check(lib.lbx_build_bouzidi_links(*args, n.value, _ptr(cells), _ptr(dirs), _ptr(wall), C.byref(n)),
          "lbx_build_bouzidi_links")
    return cells, dirs, wall


FD_VELOCITY, FD_PRESSURE, FD_LOCAL_VELOCITY, FD_LOCAL_PRESSURE = 1, 2, 3, 4
# LocalVelocity / LocalPressure with their default RLB mixin
FD_LOCAL_VELOCITY_RLB, FD_LOCAL_PRESSURE_RLB = 5, 6


NORMAL_FLAT, NORMAL_EXTERNAL_CORNER, NORMAL_INTERNAL_CORNER, NORMAL_EXTERNAL_EDGE, NORMAL_INTERNAL_EDGE = 0, 1, 2, 3, 4


def discrete_normals(material: np.ndarray, boundary: int, fluid=(1,), outside=(0,),
                     periodic=(False, False, False)):
    """computeBoundaryTypeAndNormal (geometry/discreteNormals.hh) for every cell of material
    `boundary`, through lbx_discrete_normals: returns (cells, types, normals[n, 3]) in ascending
    core-cell order; a cell matching no pattern has type NORMAL_FLAT and a zero normal."""
    mat = np.ascontiguousarray(material, dtype=np.int32)
    d = mat.ndim
    q = 9 if d == 2 else 19
    core = list(mat.shape) + [1] * (3 - d)
    fl = np.ascontiguousarray(fluid, dtype=np.int32)
    ou = np.ascontiguousarray(outside, dtype=np.int32)
    per = [int(bool(p)) for p in periodic] + [0] * (3 - len(periodic))
    n = C.c_int64()
    args = (q, _i32x3(core), _i32x3(per[:3]), _ptr(mat), int(boundary), len(fl), _ptr(fl), len(ou), _ptr(ou))
    check(lib.lbx_discrete_normals(*args, 0, None, None, None, C.byref(n)), "lbx_discrete_normals")
    cells = np.empty(n.value, np.int64)
    types = np.empty(n.value, np.int32)
    normals = np.empty((n.value, 3), np.int32)
    check(lib.lbx_discrete_normals(*args, n.value, _ptr(cells), _ptr(types), _ptr(normals), C.byref(n)),
          "lbx_discrete_normals")
    return cells, types, normals


def fd_boundaries_from_materials(material: np.ndarray, boundary: int, fluid=(1,), outside=(0,),
                                 periodic=(False, False, False)):
    """The flat-face cells of material `boundary` as boundary::set classifies them
    (discrete_normals): returns (cells, dirs, orients) of the cells whose discrete normal is flat;
    edges and corners are left out."""
    cells, types, normals = discrete_normals(material, boundary, fluid, outside, periodic)
    keep = (types == NORMAL_FLAT) & (np.abs(normals).sum(axis=1) == 1)
    cells, normals = cells[keep], normals[keep]
    dirs = np.argmax(np.abs(normals), axis=1).astype(np.int32)
    orients = normals[np.arange(len(cells)), dirs].astype(np.int32)
    return cells, dirs, orients


class BlockLattice:
    """One block lattice on one B200 (a ConcreteBlockLattice of the new platform)."""

    def __init__(self, q: int, core, periodic=(False, False, False), storage: str = "f32", device: int = 0):
        core = list(core) + [1] * (3 - len(core))
        h = C.c_void_p()
        check(lib.lbx_lattice_create(q, _i32x3(core), _i32x3(periodic), STORAGE[storage], device, C.byref(h)),
              "lbx_lattice_create")
        self._h = h
        self.q = q
        self.d = 2 if q == 9 else 3
        self.core = tuple(core)
        self.storage = storage
        self.device = device
        self.n_core = int(np.prod(core))
        self._dyn = "bgk"
        self._params = Params(1.0, 0.25, 0.12, (C.c_double * 3)(0, 0, 0))

    @classmethod
    def _borrow(cls, handle: C.c_void_p, q: int, core, storage: str, device: int) -> "BlockLattice":
        """A view of a lattice owned elsewhere (a slab of a SlabLattice): close() leaves it."""
        lat = cls.__new__(cls)
        lat._h = handle
        lat._owned = False
        lat.q = q
        lat.d = 2 if q == 9 else 3
        lat.core = tuple(core)
        lat.storage = storage
        lat.device = device
        lat.n_core = int(np.prod(core))
        lat._dyn = "bgk"
        lat._params = Params(1.0, 0.25, 0.12, (C.c_double * 3)(0, 0, 0))
        return lat

    # -- lifetime --------------------------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            if getattr(self, "_owned", True):
                lib.lbx_lattice_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def info(self) -> Info:
        i = Info()
        check(lib.lbx_get_info(self._h, C.byref(i)), "lbx_get_info")
        return i

    # -- dynamics and parameters -----------------------------------------------------------
    def define_dynamics(self, dynamics: str, omega: float | None = None, magic: float | None = None,
                        smagorinsky: float | None = None, force=None) -> None:
        self._dyn = dynamics
        if omega is not None:
            self._params.omega = omega
        if magic is not None:
            self._params.magic = magic
        if smagorinsky is not None:
            self._params.smagorinsky = smagorinsky
        if force is not None:
            f = list(force) + [0.0] * (3 - len(force))
            self._params.force = (C.c_double * 3)(*f)
        check(lib.lbx_set_dynamics(self._h, DYNAMICS[dynamics], C.byref(self._params)), "lbx_set_dynamics")

    def set_parameter(self, name: str, value) -> None:
        """setParameter<OMEGA | TRT::MAGIC | LES::SMAGORINSKY | FORCE>."""
        key = {"omega": "omega", "magic": "magic", "smagorinsky": "smagorinsky", "force": "force"}[name.lower()]
        self.define_dynamics(self._dyn, **{key: value})

    def set_dynamics_class(self, cls: int, omega: float | None = None, magic: float | None = None,
                           smagorinsky: float | None = None, force=None, remove: bool = False,
                           dynamics: str | None = None) -> None:
        """Parameters of class `cls` (1..3) of the bulk dynamics (lbx_set_dynamics_class): cells
        marked CELL_BULK_CLASS_<cls> collide with them; unspecified values are the lattice's.
        `dynamics` (a key of DYNAMICS) gives the class a dynamics of its own
        (lbx_set_dynamics_class_kind)."""
        if remove:
            check(lib.lbx_set_dynamics_class(self._h, cls, None), "lbx_set_dynamics_class")
            return
        p = Params(self._params.omega, self._params.magic, self._params.smagorinsky,
                   (C.c_double * 3)(*self._params.force))
        if omega is not None:
            p.omega = omega
        if magic is not None:
            p.magic = magic
        if smagorinsky is not None:
            p.smagorinsky = smagorinsky
        if force is not None:
            p.force = (C.c_double * 3)(*(list(force) + [0.0] * 3)[:3])
        if dynamics is not None:
            check(lib.lbx_set_dynamics_class_kind(self._h, cls, DYNAMICS[dynamics], C.byref(p)),
                  "lbx_set_dynamics_class_kind")
            return
        check(lib.lbx_set_dynamics_class(self._h, cls, C.byref(p)), "lbx_set_dynamics_class")

    def set_cell_dynamics(self, ids: np.ndarray | None) -> None:
        if ids is None:
            check(lib.lbx_set_cell_dynamics(self._h, None), "lbx_set_cell_dynamics")
            return
        a = np.ascontiguousarray(ids, dtype=np.uint8).reshape(-1)
        if a.size != self.n_core:
            raise ValueError("cell dynamics map must cover the core cells")
        check(lib.lbx_set_cell_dynamics(self._h, _ptr(a)), "lbx_set_cell_dynamics")

    def set_bouzidi_links(self, cells, dirs, wall=None) -> None:
        c = np.ascontiguousarray(cells, dtype=np.int64)
        d = np.ascontiguousarray(dirs, dtype=np.int32)
        w = None if wall is None else np.ascontiguousarray(wall, dtype=np.float64)
        check(lib.lbx_set_bouzidi_links(self._h, len(c), _ptr(c), _ptr(d), _ptr(w)), "lbx_set_bouzidi_links")

    def set_fd_boundaries(self, cells, kinds, dirs, orients, values) -> None:
        """Flat-face velocity (kind 1) / pressure (kind 2) boundary cells: the cells of
        boundary::set<InterpolatedVelocity | InterpolatedPressure>; values [n, 4] = the imposed
        velocity, or {rho, tangential velocity}."""
        c = np.ascontiguousarray(cells, dtype=np.int64)
        k = np.ascontiguousarray(kinds, dtype=np.int32)
        d = np.ascontiguousarray(dirs, dtype=np.int32)
        o = np.ascontiguousarray(orients, dtype=np.int32)
        v = np.ascontiguousarray(values, dtype=np.float64).reshape(-1, 4)
        if not (len(c) == len(k) == len(d) == len(o) == len(v)):
            raise ValueError("boundary arrays differ in length")
        check(lib.lbx_set_fd_boundaries(self._h, len(c), _ptr(c), _ptr(k), _ptr(d), _ptr(o), _ptr(v)),
              "lbx_set_fd_boundaries")

    def set_boundary_cells(self, cells, kinds, types, normals, values) -> None:
        """Velocity / pressure boundary cells with their discrete normal type (flat, external
        edge, external corner) and outward normal [n, 3]: lbx_set_boundary_cells."""
        c = np.ascontiguousarray(cells, dtype=np.int64)
        k = np.ascontiguousarray(kinds, dtype=np.int32)
        t = np.ascontiguousarray(types, dtype=np.int32)
        nn = np.ascontiguousarray(normals, dtype=np.int32).reshape(-1, 3)
        v = np.ascontiguousarray(values, dtype=np.float64).reshape(-1, 4)
        if not (len(c) == len(k) == len(t) == len(nn) == len(v)):
            raise ValueError("boundary arrays differ in length")
        check(lib.lbx_set_boundary_cells(self._h, len(c), _ptr(c), _ptr(k), _ptr(t), _ptr(nn), _ptr(v)),
              "lbx_set_boundary_cells")

    def set_bounce_back_velocity(self, cells, rho, u) -> None:
        """BounceBackVelocity cells (lbx_set_bounce_back_velocity): rho [n] (None: 1), u [n, 3]."""
        c = np.ascontiguousarray(cells, dtype=np.int64)
        r = None if rho is None else np.ascontiguousarray(rho, dtype=np.float64)
        uu = np.ascontiguousarray(u, dtype=np.float64).reshape(-1, 3)
        if len(uu) != len(c) or (r is not None and len(r) != len(c)):
            raise ValueError("bounce-back arrays differ in length")
        check(lib.lbx_set_bounce_back_velocity(self._h, len(c), _ptr(c), _ptr(r), _ptr(uu)),
              "lbx_set_bounce_back_velocity")

    def set_interpolated_boundary(self, kind: int, material: np.ndarray, boundary: int, values: np.ndarray,
                                  fluid=(1,), outside=(0,)) -> None:
        """boundary::set<InterpolatedVelocity> (kind FD_VELOCITY) or <InterpolatedPressure>
        (FD_PRESSURE) over the cells of material `boundary`; values [core cells, 4] hold the
        imposed velocity, or {rho, tangential velocity}, of each boundary cell."""
        mat = np.ascontiguousarray(material, dtype=np.int32).reshape(-1)
        v = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
        if mat.size != self.n_core or v.size != 4 * self.n_core:
            raise ValueError("material [core cells] and values [core cells, 4] expected")
        fl = np.ascontiguousarray(fluid, dtype=np.int32)
        ou = np.ascontiguousarray(outside, dtype=np.int32)
        check(lib.lbx_set_interpolated_boundary(self._h, int(kind), _ptr(mat), int(boundary), len(fl), _ptr(fl),
                                                len(ou), _ptr(ou), _ptr(v)), "lbx_set_interpolated_boundary")

    def set_bouzidi_boundary(self, material: np.ndarray, fluid: int = 1, solid=(2,), wall_velocity=None) -> None:
        mat = np.ascontiguousarray(material, dtype=np.int32).reshape(-1)
        sol = np.ascontiguousarray(solid, dtype=np.int32)
        wv = None if wall_velocity is None else np.ascontiguousarray(wall_velocity, dtype=np.float64).reshape(-1)
        check(lib.lbx_set_bouzidi_from_materials(self._h, _ptr(mat), fluid, len(sol), _ptr(sol), _ptr(wv)),
              "lbx_set_bouzidi_from_materials")

    # -- data movement -----------------------------------------------------------------------
    def set_populations(self, f: np.ndarray, stream=None) -> None:
        a = np.ascontiguousarray(f)
        if a.dtype not in (np.float64, np.float32) or a.size != self.q * self.n_core:
            raise ValueError("populations must be float64/float32 [q][core cells]")
        check(lib.lbx_upload_populations(self._h, _ptr(a), 0 if a.dtype == np.float64 else 1, _stream_ptr(stream)),
              "lbx_upload_populations")

    def get_populations(self, dtype=np.float64, stream=None, out: np.ndarray | None = None) -> np.ndarray:
        a = out if out is not None else np.empty((self.q, self.n_core), dtype=dtype)
        check(lib.lbx_download_populations(self._h, _ptr(a), 0 if a.dtype == np.float64 else 1, _stream_ptr(stream)),
              "lbx_download_populations")
        return a

    def save_checkpoint(self, stream=None) -> bytes:
        """The lattice state as a byte string (SuperLattice::save): populations of the core cells
        in logical order and the last statistics, behind a header naming the lattice's shape."""
        n = C.c_int64()
        check(lib.lbx_checkpoint_bytes(self._h, C.byref(n)), "lbx_checkpoint_bytes")
        buf = np.empty(n.value, dtype=np.uint8)
        check(lib.lbx_save_checkpoint(self._h, _ptr(buf), n.value, _stream_ptr(stream)), "lbx_save_checkpoint")
        return buf.tobytes()

    def load_checkpoint(self, data: bytes, stream=None) -> None:
        """Restores a checkpoint of a lattice with the same descriptor, storage, extent and
        periodicity (SuperLattice::load); dynamics and boundaries are the caller's set-up."""
        buf = np.frombuffer(data, dtype=np.uint8)
        check(lib.lbx_load_checkpoint(self._h, _ptr(buf), buf.size, _stream_ptr(stream)), "lbx_load_checkpoint")

    def ini_equilibrium(self, rho: np.ndarray, u: np.ndarray, stream=None) -> None:
        r = np.ascontiguousarray(rho, dtype=np.float64).reshape(-1)
        v = np.ascontiguousarray(u, dtype=np.float64).reshape(self.d, -1)
        check(lib.lbx_ini_equilibrium(self._h, _ptr(r), _ptr(v), _stream_ptr(stream)), "lbx_ini_equilibrium")

    # -- the hot path --------------------------------------------------------------------------
    def collide_and_stream(self, steps: int = 1, statistics: bool = False, stream=None) -> None:
        flags = STEP_STATISTICS if statistics else 0
        check(lib.lbx_collide_and_stream(self._h, steps, flags, _stream_ptr(stream)), "lbx_collide_and_stream")

    def post_process(self, stream=None) -> None:
        """The PostStream post-processors once (what the reference's initialize() runs)."""
        check(lib.lbx_post_process(self._h, _stream_ptr(stream)), "lbx_post_process")

    def get_statistics(self, stream=None) -> dict:
        out = (C.c_double * 4)()
        check(lib.lbx_get_statistics(self._h, out, _stream_ptr(stream)), "lbx_get_statistics")
        return {"average_rho": out[0], "average_energy": out[1], "max_u": out[2], "cells": int(out[3])}

    def compute_moments(self, stream=None):
        rho = np.empty(self.n_core, np.float64)
        u = np.empty((self.d, self.n_core), np.float64)
        check(lib.lbx_compute_moments(self._h, _ptr(rho), _ptr(u), _stream_ptr(stream)), "lbx_compute_moments")
        return rho, u

    def reduce(self, what: int, stream=None) -> np.ndarray:
        out = (C.c_double * 8)()
        check(lib.lbx_reduce(self._h, what, out, _stream_ptr(stream)), "lbx_reduce")
        n = {REDUCE_MASS_MOMENTUM: 4, REDUCE_DRAG: 3, REDUCE_RESIDUAL: 3}[what]
        return np.array(out[:n])

    def boundary_force(self, group: int = -1, stream=None) -> np.ndarray:
        """Force on the solid behind link group `group` (the index of its material in the
        `solid` list of set_bouzidi_boundary; -1: all links), lattice units, in the convention of
        the reference's SuperLatticePhysBoundaryForce3D summed over that solid."""
        out = (C.c_double * 3)()
        check(lib.lbx_boundary_force(self._h, int(group), out, _stream_ptr(stream)), "lbx_boundary_force")
        return np.array(out[:])

    def set_launch_config(self, variant: int, block_x: int = 256, block_y: int = 1,
                          cells_per_thread: int = 1) -> None:
        check(lib.lbx_set_launch_config(self._h, variant, block_x, block_y, cells_per_thread),
              "lbx_set_launch_config")

    def set_kernel_timing(self, enable: bool) -> None:
        check(lib.lbx_set_kernel_timing(self._h, 1 if enable else 0), "lbx_set_kernel_timing")

    def kernel_timing(self) -> dict:
        """Summed device ms and launch counts per kernel kind since set_kernel_timing(True)."""
        out = (C.c_double * 6)()
        check(lib.lbx_get_kernel_timing(self._h, out), "lbx_get_kernel_timing")
        return {"collision": (out[0], int(out[3])), "periodic_overlap": (out[1], int(out[4])),
                "links": (out[2], int(out[5]))}

    def autotune(self, steps: int = 20, stream=None) -> list[dict]:
        """Time every launch shape of the step kernel on this lattice's data, keep the fastest;
        the populations are left as they were.  Returns the candidates with their ms/step."""
        return _tune(lib.lbx_autotune, self._h, steps, stream, "lbx_autotune")

    def population_ptr(self, pop: int) -> tuple[int, int]:
        """(device address, shift) of population column `pop` (lbx_population_ptr)."""
        ptr = C.c_void_p()
        sh = C.c_int64()
        check(lib.lbx_population_ptr(self._h, int(pop), C.byref(ptr), C.byref(sh)), "lbx_population_ptr")
        return int(ptr.value or 0), sh.value

    def population_shift(self, pop: int) -> int:
        s = C.c_int64()
        check(lib.lbx_population_shift(self._h, pop, C.byref(s)), "lbx_population_shift")
        return s.value


def make_request(core, omega: float, lid_velocity: float, tolerance: float = 1e-6, max_steps: int = 50000,
                 dynamics: str = "bgk", magic: float = 0.25) -> EnsembleRequest:
    r = EnsembleRequest()
    r.core = (C.c_int32 * 3)(*[int(v) for v in core])
    r.dynamics = DYNAMICS[dynamics]
    r.params = Params(omega, magic, 0.0, (C.c_double * 3)(0, 0, 0))
    r.lid_velocity = lid_velocity
    r.tolerance = tolerance
    r.max_steps = max_steps
    return r


class Ensemble:
    """Many independent box cavities stepped by one persistent kernel (lbx_ensemble_*)."""

    def __init__(self, q: int = 19, storage: str = "f32", slab_bytes: int = 8 << 30, max_lattices: int = 1024,
                 device: int = 0):
        h = C.c_void_p()
        check(lib.lbx_ensemble_create(q, STORAGE[storage], slab_bytes, max_lattices, device, C.byref(h)),
              "lbx_ensemble_create")
        self._h = h
        self.q = q
        self.storage = storage
        self.max_lattices = max_lattices
        self.cells: dict[int, int] = {}

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            lib.lbx_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def footprint(self, req: EnsembleRequest) -> int:
        return Ensemble.footprint_of(self.q, self.storage, req)

    @staticmethod
    def footprint_of(q: int, storage: str, req: EnsembleRequest) -> int:
        """Slab bytes a request needs (no ensemble or device needed)."""
        b = C.c_int64()
        check(lib.lbx_ensemble_footprint(q, STORAGE[storage], C.byref(req), C.byref(b)), "lbx_ensemble_footprint")
        return b.value

    def admit(self, req: EnsembleRequest) -> int | None:
        """Slot of the admitted request, or None when the slab or the slot table is full."""
        slot = C.c_int32()
        rc = lib.lbx_ensemble_admit(self._h, C.byref(req), C.byref(slot))
        if rc == -5:
            return None
        check(rc, "lbx_ensemble_admit")
        self.cells[slot.value] = int(req.core[0]) * int(req.core[1]) * int(req.core[2])
        return slot.value

    def run(self, steps: int, stream=None) -> None:
        check(lib.lbx_ensemble_run(self._h, steps, _stream_ptr(stream)), "lbx_ensemble_run")

    def statuses(self, stream=None) -> list[tuple[int, int, float]]:
        arr = (EnsembleStatus * self.max_lattices)()
        check(lib.lbx_ensemble_statuses(self._h, arr, self.max_lattices, _stream_ptr(stream)), "lbx_ensemble_statuses")
        return [(a.state, a.steps, a.residual) for a in arr]

    def moments(self, slot: int, stream=None):
        n = self.cells[slot]
        rho = np.empty(n, np.float64)
        u = np.empty((3, n), np.float64)
        check(lib.lbx_ensemble_moments(self._h, slot, _ptr(rho), _ptr(u), _stream_ptr(stream)), "lbx_ensemble_moments")
        return rho, u

    def retire(self, slot: int) -> None:
        check(lib.lbx_ensemble_retire(self._h, slot), "lbx_ensemble_retire")
        self.cells.pop(slot, None)

    def autotune(self, steps: int = 50, stream=None) -> list[dict]:
        """Time every launch shape of the persistent kernel on the admitted lattices, keep the
        fastest; every lattice's state is left as it was."""
        return _tune(lib.lbx_ensemble_autotune, self._h, steps, stream, "lbx_ensemble_autotune")

    def set_launch_mode(self, mode: int) -> None:
        """0: one persistent kernel per run; 1: one launch per step, chained in a CUDA graph."""
        check(lib.lbx_ensemble_set_launch_mode(self._h, mode), "lbx_ensemble_set_launch_mode")

    def save_slot(self, slot: int, stream=None) -> bytes:
        """A slot's full state as bytes (pre-emption); the slot stays admitted."""
        n = C.c_int64()
        check(lib.lbx_ensemble_checkpoint_bytes(self._h, slot, C.byref(n)), "lbx_ensemble_checkpoint_bytes")
        buf = np.empty(n.value, dtype=np.uint8)
        check(lib.lbx_ensemble_save_slot(self._h, slot, _ptr(buf), n.value, _stream_ptr(stream)), "lbx_ensemble_save_slot")
        return buf.tobytes()

    def restore_slot(self, data: bytes, stream=None) -> int:
        """Admits a saved slot, which continues where it stopped; returns its new slot."""
        buf = np.frombuffer(data, dtype=np.uint8)
        slot = C.c_int32(-1)
        check(lib.lbx_ensemble_restore_slot(self._h, _ptr(buf), buf.size, C.byref(slot), _stream_ptr(stream)),
              "lbx_ensemble_restore_slot")
        core = np.frombuffer(data, dtype=np.int32, count=3, offset=16)  # the header's core extent
        self.cells[slot.value] = int(core[0]) * int(core[1]) * int(core[2])
        return slot.value

    def set_cells_per_thread(self, cells: int) -> None:
        """1 or 2 cells per thread in the tile loop (identical results)."""
        check(lib.lbx_ensemble_set_cells_per_thread(self._h, cells), "lbx_ensemble_set_cells_per_thread")

    def set_config(self, threads: int = 256, blocks_per_sm: int = 0, check_interval: int = 100) -> None:
        check(lib.lbx_ensemble_set_config(self._h, threads, blocks_per_sm, check_interval), "lbx_ensemble_set_config")


class Server:
    """The native continuous-batching request loop (lbx_server_*): admission by slab footprint,
    one ensemble run of an adaptive chunk of steps per round, retirement on convergence, all on a
    host thread of the library's own.  `engine` is an Ensemble, or a ServerEngine with its
    context for a caller-supplied engine."""

    def __init__(self, engine, min_chunk: int = 100, max_chunk: int = 500, realtime: bool = True,
                 stream=None, on_finish=None, ctx=None):
        cfg = ServerConfig(min_chunk, max_chunk, 1 if realtime else 0, 0)
        h = C.c_void_p()
        if isinstance(engine, Ensemble):
            check(lib.lbx_server_create(engine._h, engine.max_lattices, C.byref(cfg), _stream_ptr(stream),
                                        C.byref(h)), "lbx_server_create")
        else:
            check(lib.lbx_server_create_with_engine(C.byref(engine), ctx, C.byref(cfg), C.byref(h)),
                  "lbx_server_create_with_engine")
        self._h = h
        self._engine = engine  # kept alive with the callbacks it holds
        self._cb = None
        if on_finish is not None:
            self._cb = FINISH_FN(lambda _user, rec: on_finish(rec.contents))
            check(lib.lbx_server_set_finish_callback(self._h, self._cb, None), "lbx_server_set_finish_callback")

    def submit(self, requests) -> None:
        """requests: iterable of (id, arrival seconds or -1 for now, EnsembleRequest)."""
        items = list(requests)
        arr = (ServerRequest * max(len(items), 1))()
        for i, (rid, arrival, req) in enumerate(items):
            arr[i].id = rid
            arr[i].arrival = arrival
            arr[i].request = req
        check(lib.lbx_server_submit(self._h, arr, len(items)), "lbx_server_submit")

    def start(self) -> None:
        check(lib.lbx_server_start(self._h), "lbx_server_start")

    def close(self) -> None:
        check(lib.lbx_server_close(self._h), "lbx_server_close")

    def cancel(self, rid: int) -> None:
        check(lib.lbx_server_cancel(self._h, rid), "lbx_server_cancel")

    def wait(self, timeout: float = -1.0) -> bool:
        """True once the loop has ended (raises the error that stopped it, if any)."""
        fin = C.c_int32(0)
        check(lib.lbx_server_wait(self._h, timeout, C.byref(fin)), "lbx_server_wait")
        return bool(fin.value)

    def records(self, capacity: int = 4096) -> list[dict]:
        out = []
        arr = (ServerRecord * capacity)()
        while True:
            n = C.c_int32()
            check(lib.lbx_server_records(self._h, arr, capacity, C.byref(n)), "lbx_server_records")
            out += [{k: getattr(arr[i], k) for k, _ in ServerRecord._fields_} for i in range(n.value)]
            if n.value < capacity:
                return out

    def stats(self) -> dict:
        st = ServerStats()
        check(lib.lbx_server_get_stats(self._h, C.byref(st)), "lbx_server_get_stats")
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}

    def destroy(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            lib.lbx_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()


class SlabLattice:
    """One lattice cut along x into slabs stepped together with a face exchange per step
    (lbx_slabs_*), with the set-up of BlockLattice: global arrays in, global arrays out.  Each
    slab is a BlockLattice view (`slabs[k]`, first x plane `x0[k]`, extent `nx[k]`)."""

    def __init__(self, q: int, core, periodic=(False, False, False), storage: str = "f32", n_slabs: int = 2,
                 devices=None):
        core = list(core) + [1] * (3 - len(core))
        h = C.c_void_p()
        dev = None if devices is None else (C.c_int32 * n_slabs)(*[int(d) for d in devices])
        check(lib.lbx_slabs_create(q, _i32x3(core), _i32x3(periodic), STORAGE[storage], n_slabs, dev, C.byref(h)),
              "lbx_slabs_create")
        self._h = h
        self.q, self.d, self.core, self.storage = q, (2 if q == 9 else 3), tuple(core), storage
        self.periodic = tuple(bool(p) for p in (list(periodic) + [False] * 3)[:3])
        self.n_core = int(np.prod(core))
        self.plane = int(core[1]) * int(core[2])
        self.slabs: list[BlockLattice] = []
        self.x0: list[int] = []
        self.nx: list[int] = []
        for k in range(n_slabs):
            lh, x0, nx = C.c_void_p(), C.c_int32(), C.c_int32()
            check(lib.lbx_slabs_get(h, k, C.byref(lh), C.byref(x0), C.byref(nx)), "lbx_slabs_get")
            d = 0 if devices is None else int(devices[k])
            self.slabs.append(BlockLattice._borrow(lh, q, (nx.value, core[1], core[2]), storage, d))
            self.x0.append(x0.value)
            self.nx.append(nx.value)
        self._fd: list[list] = [[] for _ in range(n_slabs)]

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            for s in self.slabs:
                s._h = None
            lib.lbx_slabs_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- splitting of global arrays over core cells (x slowest) ----------------------------
    def _range(self, k: int) -> slice:
        return slice(self.x0[k] * self.plane, (self.x0[k] + self.nx[k]) * self.plane)

    def _slab_of(self, cells: np.ndarray) -> np.ndarray:
        x = np.asarray(cells, np.int64) // self.plane
        return np.searchsorted(np.asarray(self.x0), x, side="right") - 1

    # -- set-up --------------------------------------------------------------------------------
    def define_dynamics(self, dynamics: str, **kw) -> None:
        for s in self.slabs:
            s.define_dynamics(dynamics, **kw)

    def set_cell_dynamics(self, ids) -> None:
        if ids is None:
            for s in self.slabs:
                s.set_cell_dynamics(None)
            return
        a = np.ascontiguousarray(ids, dtype=np.uint8).reshape(-1)
        for k, s in enumerate(self.slabs):
            s.set_cell_dynamics(a[self._range(k)])

    def set_bouzidi_links(self, cells, dirs, wall=None) -> None:
        """Links in global core-cell numbering; each goes to the slab of its fluid cell."""
        c = np.asarray(cells, np.int64)
        d = np.asarray(dirs, np.int32)
        w = None if wall is None else np.asarray(wall, np.float64)
        owner = self._slab_of(c)
        for k, s in enumerate(self.slabs):
            sel = owner == k
            s.set_bouzidi_links(c[sel] - self.x0[k] * self.plane, d[sel], None if w is None else w[sel])

    def set_bouzidi_boundary(self, material: np.ndarray, fluid: int = 1, solid=(2,), wall_velocity=None) -> None:
        """setBouzidiBoundary over the whole lattice's material map (q = 1/2)."""
        cells, dirs, wall = build_bouzidi_links(self.q, self.core, material, fluid, solid, wall_velocity,
                                                self.periodic)
        self.set_bouzidi_links(cells, dirs, wall)

    def set_boundary_cells(self, cells, kinds, types, normals, values) -> None:
        """Velocity / pressure boundary cells in global numbering (lbx_set_boundary_cells per
        slab); each must have two planes of its slab towards every face shared with a slab."""
        c = np.asarray(cells, np.int64)
        arrs = [np.asarray(kinds, np.int32), np.asarray(types, np.int32),
                np.asarray(normals, np.int32).reshape(-1, 3), np.asarray(values, np.float64).reshape(-1, 4)]
        owner = self._slab_of(c)
        ns = len(self.slabs)
        for k in range(ns):
            sel = owner == k
            xl = c[sel] // self.plane - self.x0[k]
            lo_shared = k > 0 or (self.periodic[0] and ns > 1)
            hi_shared = k < ns - 1 or (self.periodic[0] and ns > 1)
            if (lo_shared and (xl < 2).any()) or (hi_shared and (xl > self.nx[k] - 3).any()):
                raise LbxError(-4, f"slab {k}: a boundary cell lies within two planes of a face between slabs")
            self._fd[k] = [c[sel] - self.x0[k] * self.plane] + [a[sel] for a in arrs]
            self.slabs[k].set_boundary_cells(*self._fd[k])

    def set_interpolated_boundary(self, kind: int, material: np.ndarray, boundary: int, values: np.ndarray,
                                  fluid=(1,), outside=(0,)) -> None:
        """boundary::set<InterpolatedVelocity | InterpolatedPressure> over the whole lattice:
        the cells are classified on the whole material map, then handed to their slabs (added to
        the cells set before)."""
        mat = np.asarray(material, np.int32)
        cells, types, normals = discrete_normals(mat.reshape(self.core[: self.d]), boundary, fluid, outside,
                                                 self.periodic)
        zero = ~np.abs(normals).any(axis=1)
        if zero.any() or (types < 0).any():
            raise LbxError(-4, "could not set boundary: a cell has no discrete normal")
        if kind in (FD_PRESSURE, FD_LOCAL_PRESSURE, FD_LOCAL_PRESSURE_RLB):
            keep = types == NORMAL_FLAT
            if kind in (FD_LOCAL_PRESSURE, FD_LOCAL_PRESSURE_RLB) and not keep.all():
                raise LbxError(-4, "LocalPressure: no valid discrete normal (flat faces only)")
            cells, types, normals = cells[keep], types[keep], normals[keep]
        vals = np.asarray(values, np.float64).reshape(-1, 4)[cells]
        new = [cells, np.full(len(cells), kind, np.int32), types, normals, vals]
        prev = [[f[0] + self.x0[k] * self.plane] + list(f[1:]) for k, f in enumerate(self._fd) if f]
        if prev:
            old = [np.concatenate([p[j] for p in prev]) for j in range(5)]
            stay = ~np.isin(old[0], cells)
            new = [np.concatenate([o[stay], n]) for o, n in zip(old, new)]
        order = np.argsort(new[0], kind="stable")
        self.set_boundary_cells(*[a[order] for a in new])

    def post_process(self) -> None:
        for s in self.slabs:
            s.post_process()

    # -- data movement -------------------------------------------------------------------------
    def set_populations(self, f: np.ndarray) -> None:
        a = np.asarray(f)
        for k, s in enumerate(self.slabs):
            s.set_populations(np.ascontiguousarray(a[:, self._range(k)]))

    def get_populations(self, dtype=np.float64) -> np.ndarray:
        self.synchronize()
        return np.concatenate([s.get_populations(dtype) for s in self.slabs], axis=1)

    def compute_moments(self):
        self.synchronize()
        parts = [s.compute_moments() for s in self.slabs]
        return np.concatenate([p[0] for p in parts]), np.concatenate([p[1] for p in parts], axis=1)

    # -- steps -------------------------------------------------------------------------------------
    def collide_and_stream(self, steps: int = 1, statistics: bool = False) -> None:
        check(lib.lbx_slabs_collide_and_stream(self._h, steps, STEP_STATISTICS if statistics else 0),
              "lbx_slabs_collide_and_stream")

    def synchronize(self) -> None:
        check(lib.lbx_slabs_synchronize(self._h), "lbx_slabs_synchronize")

    def get_statistics(self) -> dict:
        out = (C.c_double * 4)()
        check(lib.lbx_slabs_get_statistics(self._h, out), "lbx_slabs_get_statistics")
        return {"average_rho": out[0], "average_energy": out[1], "max_u": out[2], "cells": int(out[3])}
