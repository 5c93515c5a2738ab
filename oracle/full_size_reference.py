"""Full-size runs of the reference's own CPU code for the channel-past-a-sphere and porous-medium
configurations -- TEST INFRASTRUCTURE ONLY (records for tests/full_size_accuracy.py).

Runs the sequential FP64 reference driver (oracle/_ref/lbref_d3q27_f64_nocse, CPU_SISD with the
generic dynamics templates, see oracle/Makefile) on the same material maps the GPU runs use
(openlb_b200.configs), and writes compact records into oracle/_ref/full/:

    <case>_ref_<steps>.npz   the boundary-force history on the sphere (channel), the statistics of
                             the last step, and the moment fields (rho, u) on probe sets: every
                             4th cell along each axis, and full planes through the obstacle.

    python oracle/full_size_reference.py check            # OpenMP build against the sequential one
    python oracle/full_size_reference.py channel STEPS
    python oracle/full_size_reference.py porous STEPS

The sequential build is used although it runs on one core: `check` shows that the reference's
OpenMP build (oracle/_ref/lbref_d3q27_f64_omp) does not reproduce its own results once halfway
bounce-back links are present -- two runs of the same 32^3 porous case differ after three steps,
with the set-up on one thread as well -- while it agrees bit for bit without the links and when
run on one thread.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF = HERE / "_ref"
RECORDS = REF / "full"      # finished records
SCRATCH = HERE.parent / "_scratch"  # the runs' working files (large; neither committed nor sent to a GPU box)
sys.path.insert(0, str(HERE.parent))

from openlb_b200 import configs  # noqa: E402  (material maps and profiles only; no GPU work)

CHANNEL = {"extent": (512, 128, 128), "center": (128, 64, 64), "d": 24.0, "u_peak": 0.04, "re": 50.0}
POROUS = {"n": 384, "seed": 7, "porosity": 0.6, "nu": 0.05, "force": 1e-6, "cs": 0.12}


def channel_args(steps: int) -> tuple[np.ndarray, list[str]]:
    c = CHANNEL
    mat = configs.channel_materials(c["extent"], c["center"], c["d"])
    nu = c["u_peak"] * c["d"] / c["re"]
    omega = 1.0 / (3 * nu + 0.5)
    args = ["--n", *map(str, c["extent"]), "--dyn", "trt", "--omega", repr(omega), "--magic", "0.25",
            "--ivel", "3", "--poiseuille", repr(c["u_peak"]), "--ipres", "4", "--rho", "1",
            "--bounceback", "2", "--bouzidi", "5", "--force-mat", "5", "--force-every", "500",
            "--init", "rest", "--steps", str(steps)]
    return mat, args


def porous_args(steps: int) -> tuple[np.ndarray, list[str]]:
    p = POROUS
    solid = configs.porous_spheres(p["n"], p["seed"], p["porosity"])
    mat = np.where(solid, 2, 1).astype(np.int32)
    omega = 1.0 / (3 * p["nu"] + 0.5)
    args = ["--n", *([str(p["n"])] * 3), "--periodic", "1", "1", "1", "--dyn", "fsmag", "--omega", repr(omega),
            "--cs", repr(p["cs"]), "--force", repr(p["force"]), "0", "0", "--bouzidi", "2", "--init", "rest",
            "--steps", str(steps)]
    return mat, args


def probes(shape, planes) -> np.ndarray:
    """Flat indices of the probe set: every 4th cell along each axis plus the given planes
    (axis, index)."""
    idx = np.arange(int(np.prod(shape))).reshape(shape)
    sel = [idx[::4, ::4, ::4].reshape(-1)]
    for axis, k in planes:
        sel.append(np.take(idx, k, axis=axis).reshape(-1))
    return np.unique(np.concatenate(sel))


def run(case: str, steps: int, threads: int | None = None) -> Path:
    mat, args = channel_args(steps) if case == "channel" else porous_args(steps)
    exe = REF / "lbref_d3q27_f64_nocse"
    RECORDS.mkdir(parents=True, exist_ok=True)
    SCRATCH.mkdir(parents=True, exist_ok=True)
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    with tempfile.TemporaryDirectory(dir=SCRATCH) as tmp:
        prefix = str(Path(tmp) / "r")
        mat.tofile(prefix + ".in.mat")
        t0 = time.time()
        subprocess.run([str(exe), "geo", *args, "--mat", prefix + ".in.mat", "--no-pops", "--moments", "--stats",
                        "--out", prefix], check=True, env=env, stdout=subprocess.DEVNULL)
        sec = time.time() - t0
        n = mat.size
        mom = np.fromfile(prefix + ".mom.bin", dtype=np.float64).reshape(4, n)
        stats = np.loadtxt(prefix + ".stats.txt", ndmin=2)
        meta = json.loads(Path(prefix + ".json").read_text())
        force = np.loadtxt(prefix + ".force.txt", ndmin=2) if Path(prefix + ".force.txt").exists() else np.zeros((0, 4))
    if case == "channel":
        c = CHANNEL
        planes = [(2, c["center"][2]), (1, c["center"][1]), (0, c["center"][0] + int(c["d"]))]
    else:
        planes = [(2, POROUS["n"] // 2)]
    sel = probes(mat.shape, planes)
    fluid = np.isin(mat.reshape(-1), (1,))
    out = RECORDS / f"{case}_ref_{steps}.npz"
    np.savez_compressed(out, cells=sel, rho=mom[0, sel], u=mom[1:, sel], fluid=fluid[sel], force=force,
                        stats=stats[-1], mean_u=mom[1:, fluid].mean(axis=1), mean_rho=mom[0, fluid].mean(),
                        seconds=sec, meta=json.dumps({**meta, "case": case, "threads": threads or os.cpu_count()}))
    return out


def check() -> None:
    """Whether the OpenMP FP64 build gives the sequential FP64 build's bits (a 32^3 porous case
    and a reduced channel); prints the outcome of each."""
    cases = []
    solid = configs.porous_spheres(32, 3, 0.6, 4.0, 10.0)
    cases.append((np.where(solid, 2, 1).astype(np.int32),
                  ["--n", "32", "32", "32", "--periodic", "1", "1", "1", "--dyn", "fsmag", "--omega", "1.5",
                   "--cs", "0.12", "--force", "1e-4", "0", "0", "--bouzidi", "2", "--steps", "30"]))
    cmat = configs.channel_materials((40, 20, 18), (12, 10, 9), 6.0)
    cases.append((cmat, ["--n", "40", "20", "18", "--dyn", "trt", "--omega", "1.6", "--magic", "0.25", "--ivel", "3",
                         "--poiseuille", "0.04", "--ipres", "4", "--rho", "1", "--bounceback", "2", "--bouzidi", "5",
                         "--steps", "30"]))
    for mat, args in cases:
        outs = []
        for exe in ("lbref_d3q27_f64_nocse", "lbref_d3q27_f64_omp"):
            with tempfile.TemporaryDirectory() as tmp:
                prefix = str(Path(tmp) / "r")
                mat.tofile(prefix + ".in.mat")
                subprocess.run([str(REF / exe), "geo", *args, "--mat", prefix + ".in.mat", "--out", prefix],
                               check=True, stdout=subprocess.DEVNULL)
                outs.append(np.fromfile(prefix + ".fS.bin", dtype=np.float64))
        same = np.array_equal(outs[0], outs[1])
        print(f"{args[1:4]}: OpenMP build bitwise equal to the sequential build: {same}")


if __name__ == "__main__":
    if sys.argv[1] == "check":
        check()
    else:
        print(run(sys.argv[1], int(sys.argv[2]), int(sys.argv[3]) if len(sys.argv) > 3 else None))
