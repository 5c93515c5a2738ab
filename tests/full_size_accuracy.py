"""Accuracy of the full-size channel-past-a-sphere and porous-medium configurations on the GPU,
against the reference's own FP64 run and between the storage forms -- TEST INFRASTRUCTURE
(a script run on a B200, not a pytest module; its summary is committed under profiles/).

    python tests/full_size_accuracy.py channel [--steps 20000] [--ref-steps 5000]
    python tests/full_size_accuracy.py porous  [--steps 10000] [--ref-steps 1000]

1. FP64 on the GPU is run to the step count of the reference record
   (oracle/_ref/full/<case>_ref_<ref-steps>.npz, made by oracle/full_size_reference.py) and
   compared with it on the record's probe cells (fluid cells only: rho and u of a fluid cell are
   sum f + 1 and j / rho on both sides; the forced dynamics add F / 2) and, for the channel,
   through the boundary force on the sphere every 500 steps.
2. The FP64 run goes on to `--steps`; it is the FP64 oracle of the storage forms.
3. FP32, FP16 and BF16 deviation storage run the same steps; their velocity fields are compared
   with FP64 over all fluid cells (relative L2 and L_inf of u), and their drag coefficient
   (channel: C_d = 2 F_x / (rho U^2 pi d^2 / 4), U = the inlet peak) or permeability (porous:
   k = nu <u_x> / F_x, <u_x> the x velocity averaged over the whole box, solid cells counted as
   zero) with the FP64 value.
Prints one JSON object.
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

from openlb_b200 import configs, lbx  # noqa: E402

RECORDS = ROOT / "oracle" / "_ref" / "full"


def build(case: str, storage: str):
    import full_size_reference as R
    if case == "channel":
        c = R.CHANNEL
        lat, mat = configs.channel_sphere(storage, c["extent"], c["u_peak"], c["d"], c["re"], c["center"])
        return lat, mat, {"group": 0, "nu": c["u_peak"] * c["d"] / c["re"]}
    p = R.POROUS
    solid = configs.porous_spheres(p["n"], p["seed"], p["porosity"])
    lat = configs.porous_medium(solid, storage, nu=p["nu"], force=p["force"], cs=p["cs"])
    mat = np.where(solid, 2, 1).astype(np.int32)
    return lat, mat, {"nu": p["nu"], "force": p["force"]}


def moments(lat):
    rho, u = lat.compute_moments()
    return rho, u


def run_form(case: str, storage: str, steps: int, ref_steps: int | None, rec):
    import torch
    lat, mat, info = build(case, storage)
    fluid = mat.reshape(-1) == 1
    out = {"storage": storage, "steps": steps}
    forces = []
    done = 0
    t_steps = 0.0

    def advance(k):
        nonlocal done, t_steps
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        lat.collide_and_stream(k)
        torch.cuda.synchronize()
        t_steps += time.perf_counter() - t0
        done += k

    if ref_steps:
        # to the reference's step count, with the force history on its schedule
        every = 500 if case == "channel" else ref_steps
        while done < ref_steps:
            advance(min(every, ref_steps - done))
            if case == "channel":
                forces.append([done, *lat.boundary_force(info["group"])])
        rho, u = moments(lat)
        sel = rec["cells"][rec["fluid"]]
        du = u[:, sel] - rec["u"][:, rec["fluid"]]
        out["vs_reference"] = {
            "steps": ref_steps,
            "probe_cells": int(len(sel)),
            "u_max_abs": float(np.abs(du).max()),
            "u_max_rel": float(np.abs(du).max() / np.abs(rec["u"][:, rec["fluid"]]).max()),
            "rho_max_abs": float(np.abs(rho[sel] - rec["rho"][rec["fluid"]]).max()),
            "mean_u_rel": (np.abs(u[:, fluid].mean(axis=1) - rec["mean_u"]) / np.abs(rec["mean_u"]).max()).tolist(),
        }
        if case == "channel" and len(rec["force"]):
            f_ref = np.asarray(rec["force"])[:, 1:4]
            f_gpu = np.asarray(forces)[: len(f_ref), 1:4]
            out["vs_reference"]["force_max_rel"] = float(np.abs(f_gpu - f_ref).max() / np.abs(f_ref).max())
            out["vs_reference"]["force_ref_last"] = f_ref[-1].tolist()
            out["vs_reference"]["force_gpu_last"] = f_gpu[-1].tolist()
    every = 1000
    while done < steps:
        advance(min(every, steps - done))
        if case == "channel":
            forces.append([done, *lat.boundary_force(info["group"])])
    rho, u = moments(lat)
    out["mlups"] = lat.n_core * done / t_steps / 1e6
    out["seconds"] = t_steps
    lat.close()
    return out, rho, u, fluid, np.asarray(forces), info


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["channel", "porous"])
    ap.add_argument("--steps", type=int)
    ap.add_argument("--ref-steps", type=int)
    ap.add_argument("--forms", nargs="+", default=["f32", "f16dev", "bf16dev"])
    a = ap.parse_args(argv)
    steps = a.steps or (20000 if a.case == "channel" else 10000)
    ref_steps = a.ref_steps or (5000 if a.case == "channel" else 1000)
    rec_path = RECORDS / f"{a.case}_ref_{ref_steps}.npz"
    rec = dict(np.load(rec_path)) if rec_path.exists() else None
    result = {"case": a.case, "steps": steps, "reference_record": rec_path.name if rec else None}
    if rec is not None:
        result["reference_seconds"] = float(rec["seconds"])
    f64, rho64, u64, fluid, forces64, info = run_form(a.case, "f64", steps, ref_steps if rec else None, rec)
    result["f64"] = f64
    result["f64"]["u_scale"] = float(np.abs(u64[:, fluid]).max())
    if a.case == "channel":
        c_d = lambda fx: configs.drag_coefficient(fx, 0.04, 24.0)  # noqa: E731
        result["f64"]["drag_coefficient"] = c_d(forces64[-1, 1])
        result["f64"]["force_last"] = forces64[-1, 1:4].tolist()
    else:
        k64 = info["nu"] * u64[0, fluid].sum() / fluid.size / info["force"]
        result["f64"]["permeability"] = float(k64)
        result["f64"]["porosity"] = float(fluid.mean())
    for form in a.forms:
        r, rho, u, _, forces, _ = run_form(a.case, form, steps, None, None)
        du = u[:, fluid] - u64[:, fluid]
        r["u_l2_vs_f64"] = float(np.sqrt((du ** 2).sum() / (u64[:, fluid] ** 2).sum()))
        r["u_linf_vs_f64"] = float(np.abs(du).max() / np.abs(u64[:, fluid]).max())
        r["rho_max_abs_vs_f64"] = float(np.abs(rho[fluid] - rho64[fluid]).max())
        if a.case == "channel":
            cd = configs.drag_coefficient(forces[-1, 1], 0.04, 24.0)
            r["drag_coefficient"] = cd
            r["drag_coefficient_rel_vs_f64"] = abs(cd - result["f64"]["drag_coefficient"]) / abs(
                result["f64"]["drag_coefficient"])
        else:
            k = info["nu"] * u[0, fluid].sum() / fluid.size / info["force"]
            r["permeability"] = float(k)
            r["permeability_rel_vs_f64"] = abs(k - result["f64"]["permeability"]) / abs(result["f64"]["permeability"])
        result[form] = r
        print(json.dumps({form: r}), file=sys.stderr, flush=True)
    print(json.dumps(result))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
