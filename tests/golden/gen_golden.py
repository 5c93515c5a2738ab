"""Generate the golden fixtures of tests/golden/ from the reference's own CPU code.

Runs the reference drivers built by `make -C oracle ref` (oracle/ref_driver.cpp compiled
against the reference sources: sequential CPU_SISD, FP64 with and without the generated CSE
kernels, and FP32) on small seeded cases and stores, per case, the core-cell populations
after initialize() (f0) and after `steps` steps (fS), the material map and the per-step
lattice statistics.  Needs the reference tree (this container only); the fixtures it writes
are committed and are all the tests need.

    python tests/golden/gen_golden.py            # all cases
    python tests/golden/gen_golden.py NAME ...   # selected cases

The "geo" cases write their material map (geo_box, geo_channel) to a file the driver reads, and
keep the imposed boundary values (vals [cells, 4]), the reference's classification of every
boundary cell it set up (bclass rows {cell, kind, normal type, n0, n1, n2}) and the boundary
force on the sphere over time (force rows {step, Fx, Fy, Fz}) beside the populations.
"""
from __future__ import annotations

import json
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF = HERE.parent.parent / "oracle" / "_ref"

P3 = ["--n", "6", "7", "8"]
P2 = ["--n", "12", "10"]
RND = ["--init", "random", "--amp", "0.04", "--u0", "0.08"]
FORCE3 = ["--force", "1e-3", "-2e-4", "5e-4"]
FORCE2 = ["--force", "1e-3", "-2e-4"]

# name: (binary suffix, case, args)
CASES: dict[str, tuple[str, str, list[str]]] = {}
for q, geo in ((9, P2), (19, P3), (27, P3)):
    FORCE = FORCE2 if q == 9 else FORCE3
    for dyn, extra in (("bgk", ["--omega", "1.7"]), ("trt", ["--omega", "1.6", "--magic", "0.25"]),
                       ("smag", ["--omega", "1.95", "--cs", "0.12"]), ("fbgk", ["--omega", "1.3", *FORCE]),
                       ("fsmag", ["--omega", "1.95", "--cs", "0.12", *FORCE])):
        args = ["periodic", *geo, "--dyn", dyn, *extra, *RND, "--steps", "20", "--seed", str(q)]
        CASES[f"periodic_d{'2' if q == 9 else '3'}q{q}_{dyn}_f64"] = (f"d{'2' if q == 9 else '3'}q{q}_f64_nocse", args[0], args[1:])
        CASES[f"periodic_d{'2' if q == 9 else '3'}q{q}_{dyn}_f64cse"] = (f"d{'2' if q == 9 else '3'}q{q}_f64", args[0], args[1:])
        CASES[f"periodic_d{'2' if q == 9 else '3'}q{q}_{dyn}_f32"] = (f"d{'2' if q == 9 else '3'}q{q}_f32", args[0], args[1:])

CASES.update({
    # lid-driven cavities: halfway bounce-back walls (q = 1/2 Bouzidi) + moving lid
    "cavity_d2q9_bgk_f64": ("d2q9_f64_nocse", "cavity", ["--n", "16", "14", "--dyn", "bgk", "--omega", "1.2",
                                                          "--ulid", "0.1", "--init", "rest", "--steps", "150"]),
    "cavity_d2q9_bgk_f32": ("d2q9_f32", "cavity", ["--n", "16", "14", "--dyn", "bgk", "--omega", "1.2",
                                                    "--ulid", "0.1", "--init", "rest", "--steps", "150"]),
    "cavity_d3q19_bgk_f64": ("d3q19_f64_nocse", "cavity", ["--n", "8", "9", "7", "--dyn", "bgk", "--omega", "1.4",
                                                            "--ulid", "0.05", "--init", "rest", "--steps", "60"]),
    "cavity_d3q19_trt_f64": ("d3q19_f64_nocse", "cavity", ["--n", "8", "9", "7", "--dyn", "trt", "--omega", "1.4",
                                                            "--ulid", "0.05", "--init", "rest", "--steps", "60"]),
    "cavity_d3q27_smag_f64": ("d3q27_f64_nocse", "cavity", ["--n", "7", "8", "6", "--dyn", "smag", "--omega", "1.9",
                                                             "--cs", "0.12", "--ulid", "0.05", "--init", "rest",
                                                             "--steps", "60"]),
    # bounce-back dynamics (collision::Revert) on the walls
    "cavity_d3q19_bb_f64": ("d3q19_f64_nocse", "cavity", ["--n", "8", "9", "7", "--dyn", "bgk", "--omega", "1.4",
                                                           "--walls", "bounceback", *RND, "--steps", "40"]),
    "cavity_d2q9_bb_f64": ("d2q9_f64_nocse", "cavity", ["--n", "12", "11", "--dyn", "trt", "--omega", "1.4",
                                                         "--walls", "bounceback", *RND, "--steps", "40"]),
    # periodic porous media: random solid cells with halfway bounce-back, body force
    "porous_d3q19_fbgk_f64": ("d3q19_f64_nocse", "porous", ["--n", "8", "9", "10", "--dyn", "fbgk", "--omega", "1.5",
                                                             "--force", "1e-4", "0", "0", "--solid-frac", "0.25",
                                                             *RND, "--steps", "40"]),
    "porous_d3q27_fsmag_f64": ("d3q27_f64_nocse", "porous", ["--n", "8", "9", "10", "--dyn", "fsmag", "--omega", "1.9",
                                                              "--cs", "0.12", "--force", "1e-4", "0", "0",
                                                              "--solid-frac", "0.25", *RND, "--steps", "40"]),
    "porous_d2q9_trt_f64": ("d2q9_f64_nocse", "porous", ["--n", "14", "12", "--dyn", "trt", "--omega", "1.5",
                                                          "--solid-frac", "0.2", *RND, "--steps", "40"]),
    # channels with a velocity inlet and a pressure outlet on flat faces (InterpolatedVelocity /
    # InterpolatedPressure), periodic across, bounce-back layers behind the open faces
    "channel_d2q9_bgk_f64": ("d2q9_f64_nocse", "channel", ["--n", "14", "11", "--dyn", "bgk", "--omega", "1.3",
                                                            *RND, "--u0", "0.05", "--steps", "200"]),
    "channel_d3q19_bgk_f64": ("d3q19_f64_nocse", "channel", ["--n", "12", "10", "8", "--dyn", "bgk", "--omega", "1.2",
                                                              *RND, "--u0", "0.05", "--steps", "60"]),
    "channel_d3q19_trt_f64": ("d3q19_f64_nocse", "channel", ["--n", "12", "10", "8", "--dyn", "trt", "--omega", "1.6",
                                                              "--magic", "0.25", *RND, "--u0", "0.05", "--steps", "60"]),
    "channel_d3q27_bgk_f64": ("d3q27_f64_nocse", "channel", ["--n", "10", "8", "6", "--dyn", "bgk", "--omega", "1.5",
                                                              *RND, "--u0", "0.05", "--steps", "40"]),
    "channel_d3q19_bgk_f32": ("d3q19_f32", "channel", ["--n", "12", "10", "8", "--dyn", "bgk", "--omega", "1.2",
                                                        *RND, "--u0", "0.05", "--steps", "60"]),
    # the 2D cavity at its full size: 128^2 fluid cells, nu = 0.1 * 128 / 100, lid 0.1, 20 000
    # steps from rest (statistics kept every 100th step and the last)
    "full_cavity_d2q9_bgk_128_f64": ("d2q9_f64_nocse", "cavity", ["--n", "128", "128", "--dyn", "bgk",
                                                                   "--omega", str(1.0 / (3 * 0.128 + 0.5)),
                                                                   "--ulid", "0.1", "--init", "rest",
                                                                   "--steps", "20000"]),
    # ConstRhoBGK (the bulk dynamics of the cavity2d example): a periodic lattice whose random
    # initial density averages below 1, which the dynamics pulls back to 1, and a cavity
    "periodic_d2q9_constrho_f64": ("d2q9_f64_nocse", "periodic", [*P2, "--dyn", "constrho", "--omega", "1.7", *RND,
                                                                  "--steps", "20", "--seed", "9"]),
    "periodic_d2q9_constrho_f32": ("d2q9_f32", "periodic", [*P2, "--dyn", "constrho", "--omega", "1.7", *RND,
                                                            "--steps", "20", "--seed", "9"]),
    "periodic_d3q19_constrho_f64": ("d3q19_f64_nocse", "periodic", [*P3, "--dyn", "constrho", "--omega", "1.5",
                                                                    *RND, "--steps", "20", "--seed", "19"]),
    "cavity_d2q9_constrho_f64": ("d2q9_f64_nocse", "cavity", ["--n", "16", "14", "--dyn", "constrho", "--omega", "1.2",
                                                              "--ulid", "0.1", "--init", "rest", "--steps", "150"]),
    # Taylor-Green vortex (the benchmark's initial condition), small
    "tgv_d3q19_bgk_f64": ("d3q19_f64_nocse", "periodic", ["--n", "16", "16", "16", "--dyn", "bgk",
                                                           "--omega", str(1.0 / (3 * 0.01 + 0.5)), "--init", "tgv",
                                                           "--u0", "0.05", "--steps", "50"]),
    "tgv_d3q19_bgk_f32": ("d3q19_f32", "periodic", ["--n", "16", "16", "16", "--dyn", "bgk",
                                                     "--omega", str(1.0 / (3 * 0.01 + 0.5)), "--init", "tgv",
                                                     "--u0", "0.05", "--steps", "50"]),
})



# ---- material maps of the "geo" cases (materials from a file, the reference's own setters) ----
def geo_box(shape, lid=True):
    """A closed box: the outer layer is material 2, the top layer along y (edges and corners
    included) material 3 when `lid`, the inside fluid (1)."""
    mat = np.full(shape, 2, np.int32)
    inner = tuple(slice(1, s - 1) for s in shape)
    mat[inner] = 1
    if lid:
        mat[:, -1, ...] = 3
    return mat


def geo_step(shape, block):
    """A closed box with a block cut out of one corner of its inside (slices `block`), so that
    the fluid has internal (concave) edges and corners: the fluid (1) is the inside less the
    block, the cells next to it (diagonals included) the walls (2; 3 on the top layer along y,
    the lid), every other cell outside (0)."""
    import itertools
    fluid = np.zeros(shape, bool)
    fluid[tuple(slice(1, s - 1) for s in shape)] = True
    fluid[block] = False
    pad = np.pad(fluid, 1)
    near = np.zeros(shape, bool)
    for off in itertools.product((-1, 0, 1), repeat=len(shape)):
        if any(off):
            near |= pad[tuple(slice(1 + o, 1 + o + s) for o, s in zip(off, shape))]
    mat = np.zeros(shape, np.int32)
    mat[fluid] = 1
    wall = ~fluid & near
    mat[wall] = 2
    top = np.zeros(shape, bool)
    top[:, -1, ...] = True
    mat[wall & top] = 3
    return mat


def geo_two_dynamics(shape):
    """A periodic box of fluid (material 1) with a block in its middle of material 6, which
    carries a second fluid dynamics (--bgk-mat 6)."""
    mat = np.ones(shape, np.int32)
    inner = tuple(slice(s // 3, s - s // 3) for s in shape)
    mat[inner] = 6
    return mat


def geo_channel(shape, sphere):
    """The channel past a sphere of the full-size configuration (openlb_b200.configs.
    channel_materials) at a reduced size: sphere = (centre x, y, z, radius)."""
    sys.path.insert(0, str(HERE.parent.parent))
    from openlb_b200.configs import channel_materials
    cx, cy, cz, r = sphere
    return channel_materials(tuple(shape), (cx, cy, cz), 2 * r)


GEO = {
    # cavity2d's setup: InterpolatedVelocity on every wall (flat faces and external corners),
    # the lid the top row including its corners
    "geo_cavity_d2q9_ivel_bgk_f64": ("d2q9_f64_nocse", (14, 12), ["--dyn", "bgk", "--omega", "1.3", "--ivel", "2",
                                                                  "--ivel-lid", "3", "--ulid", "0.1", "--steps", "150"]),
    # the same set-up from rest, as examples/laminar/cavity2d starts it (the C++ example
    # openlb_b200/platform/cavity2d.cpp runs it through the C++ host layer)
    "geo_cavity2d_d2q9_ivel_bgk_rest_f64": ("d2q9_f64_nocse", (34, 34), ["--dyn", "bgk", "--omega", "1.6", "--ivel",
                                                                         "2", "--ivel-lid", "3", "--ulid", "0.1",
                                                                         "--init", "rest", "--steps", "400"]),
    "geo_cavity_d2q9_ivel_bgk_f32": ("d2q9_f32", (14, 12), ["--dyn", "bgk", "--omega", "1.3", "--ivel", "2",
                                                            "--ivel-lid", "3", "--ulid", "0.1", "--steps", "150"]),
    "geo_cavity_d2q9_ivel_constrho_f64": ("d2q9_f64_nocse", (14, 12), ["--dyn", "constrho", "--omega", "1.3",
                                                                       "--ivel", "2", "--ivel-lid", "3", "--ulid",
                                                                       "0.1", "--steps", "150"]),
    "geo_cavity_d2q9_ivel_rnd_f64": ("d2q9_f64_nocse", (13, 11), ["--dyn", "trt", "--omega", "1.5", "--magic", "0.25",
                                                                  "--ivel", "2", "--ivel-lid", "3", "--ulid", "0.08",
                                                                  *RND, "--steps", "80"]),
    # bounce-back walls and a lid of BounceBackVelocity (Revert + Nguyen-Ladd correction)
    "geo_cavity_d2q9_bbvel_f64": ("d2q9_f64_nocse", (14, 12), ["--dyn", "bgk", "--omega", "1.3", "--bounceback", "2",
                                                               "--bbvel", "3", "--ulid", "0.1", "--steps", "150"]),
    "geo_cavity_d3q19_bbvel_f64": ("d3q19_f64_nocse", (9, 8, 10), ["--dyn", "trt", "--omega", "1.5", "--magic", "0.25",
                                                                   "--bounceback", "2", "--bbvel", "3", "--ulid",
                                                                   "0.05", *RND, "--steps", "60"]),
    # a 3D cavity with InterpolatedVelocity on every wall: flat faces, external edges and corners
    "geo_cavity_d3q19_ivel_bgk_f64": ("d3q19_f64_nocse", (9, 8, 10), ["--dyn", "bgk", "--omega", "1.4", "--ivel", "2",
                                                                      "--ivel-lid", "3", "--ulid", "0.05", *RND,
                                                                      "--steps", "60"]),
    "geo_cavity_d3q27_ivel_trt_f64": ("d3q27_f64_nocse", (8, 9, 7), ["--dyn", "trt", "--omega", "1.6", "--magic",
                                                                     "0.25", "--ivel", "2", "--ivel-lid", "3",
                                                                     "--ulid", "0.05", "--steps", "80"]),
    "geo_cavity_d3q19_ivel_bgk_f32": ("d3q19_f32", (9, 8, 10), ["--dyn", "bgk", "--omega", "1.4", "--ivel", "2",
                                                                "--ivel-lid", "3", "--ulid", "0.05", "--steps", "60"]),
    # the channel past a sphere at reduced size: D3Q27 TRT (magic 1/4), RectanglePoiseuille3D inlet
    # (peak 0.04), pressure outlet, bounce-back side walls, halfway bounce-back sphere, force on the
    # sphere.  The side walls carry BounceBack dynamics: with no dynamics on the wall cells, the
    # populations the wall cells pass on to the inlet and outlet cells along the faces come from
    # the block's padding, whose content in the reference is whatever the periodic-shift storage
    # rotates into it, so the result would depend on the padding layout.
    "geo_channel_d3q27_trt_f64": ("d3q27_f64_nocse", (26, 14, 14), ["--dyn", "trt", "--omega", "1.6", "--magic",
                                                                    "0.25", "--ivel", "3", "--poiseuille", "0.04",
                                                                    "--ipres", "4", "--rho", "1", "--bounceback", "2",
                                                                    "--bouzidi", "5", "--force-mat", "5",
                                                                    "--force-every", "10",
                                                                    "--steps", "120"]),
    "geo_channel_d3q27_trt_f32": ("d3q27_f32", (26, 14, 14), ["--dyn", "trt", "--omega", "1.6", "--magic", "0.25",
                                                              "--ivel", "3", "--poiseuille", "0.04", "--ipres", "4",
                                                              "--rho", "1", "--bounceback", "2", "--bouzidi", "5",
                                                              "--force-mat", "5",
                                                              "--force-every", "10", "--steps", "120"]),
    "geo_channel_d3q19_bgk_rnd_f64": ("d3q19_f64_nocse", (20, 12, 11), ["--dyn", "bgk", "--omega", "1.3", "--ivel",
                                                                        "3", "--poiseuille", "0.05", "--ipres", "4",
                                                                        "--rho", "0.99", "--bounceback", "2", "--bouzidi", "5",
                                                                        "--force-mat", "5", "--force-every", "5",
                                                                        *RND, "--steps", "60"]),
    # boundary::LocalVelocity / LocalPressure with BGK mixed in (cavity3dBenchmark's walls): flat
    # cells regularised in their collision (CombinedRLBdynamics), edges and corners as for the
    # interpolated boundary
    "geo_cavity_d3q19_lvel_bgk_f64": ("d3q19_f64_nocse", (9, 8, 10), ["--dyn", "bgk", "--omega", "1.4", "--ivel", "2",
                                                                      "--ivel-lid", "3", "--ulid", "0.05", "--local",
                                                                      *RND, "--steps", "60"]),
    "geo_cavity_d2q9_lvel_bgk_f64": ("d2q9_f64_nocse", (14, 12), ["--dyn", "bgk", "--omega", "1.3", "--ivel", "2",
                                                                  "--ivel-lid", "3", "--ulid", "0.1", "--local",
                                                                  "--steps", "150"]),
    "geo_cavity_d3q27_lvel_trt_f64": ("d3q27_f64_nocse", (8, 9, 7), ["--dyn", "trt", "--omega", "1.6", "--magic",
                                                                     "0.25", "--ivel", "2", "--ivel-lid", "3",
                                                                     "--ulid", "0.05", "--local", "--steps", "80"]),
    "geo_channel_d3q19_lvel_lpres_f64": ("d3q19_f64_nocse", (20, 12, 11), ["--dyn", "bgk", "--omega", "1.3", "--ivel",
                                                                           "3", "--poiseuille", "0.05", "--ipres", "4",
                                                                           "--rho", "0.99", "--bounceback", "2",
                                                                           "--bouzidi", "5", "--local", *RND,
                                                                           "--steps", "60"]),
    # a cavity with a block cut out of a corner: internal (concave) edges and corners of the
    # velocity boundary (CombinedRLBdynamics with the inner edge / corner momenta), beside flat
    # faces and external edges and corners
    "geo_step_d2q9_ivel_bgk_f64": ("d2q9_f64_nocse", (14, 12), ["--dyn", "bgk", "--omega", "1.3", "--ivel", "2",
                                                                "--ivel-lid", "3", "--ulid", "0.1", "--steps", "150"]),
    "geo_step_d3q19_ivel_bgk_f64": ("d3q19_f64_nocse", (12, 11, 10), ["--dyn", "bgk", "--omega", "1.4", "--ivel", "2",
                                                                      "--ivel-lid", "3", "--ulid", "0.05", *RND,
                                                                      "--steps", "60"]),
    "geo_step_d3q27_ivel_trt_f64": ("d3q27_f64_nocse", (11, 10, 9), ["--dyn", "trt", "--omega", "1.6", "--magic",
                                                                     "0.25", "--ivel", "2", "--ivel-lid", "3",
                                                                     "--ulid", "0.05", "--steps", "80"]),
    "geo_step_d3q19_lvel_bgk_f64": ("d3q19_f64_nocse", (12, 11, 10), ["--dyn", "bgk", "--omega", "1.4", "--ivel", "2",
                                                                      "--ivel-lid", "3", "--ulid", "0.05", "--local",
                                                                      *RND, "--steps", "60"]),
    "geo_step_d3q19_ivel_bgk_f32": ("d3q19_f32", (12, 11, 10), ["--dyn", "bgk", "--omega", "1.4", "--ivel", "2",
                                                                "--ivel-lid", "3", "--ulid", "0.05", "--steps", "60"]),
    # LocalVelocity / LocalPressure with their default mixed-in dynamics, RLBdynamics: the flat
    # cells, internal edges and corners regularised twice (CombinedRLBdynamics, then the RLB
    # collision), the external edges and corners collided by RLB with the fixed-velocity momenta
    "geo_cavity_d3q19_lrlb_bgk_f64": ("d3q19_f64_nocse", (9, 8, 10), ["--dyn", "bgk", "--omega", "1.4", "--ivel", "2",
                                                                      "--ivel-lid", "3", "--ulid", "0.05",
                                                                      "--local-rlb", *RND, "--steps", "60"]),
    "geo_cavity_d2q9_lrlb_bgk_f64": ("d2q9_f64_nocse", (14, 12), ["--dyn", "bgk", "--omega", "1.3", "--ivel", "2",
                                                                  "--ivel-lid", "3", "--ulid", "0.1", "--local-rlb",
                                                                  "--steps", "150"]),
    "geo_step_d3q27_lrlb_trt_f64": ("d3q27_f64_nocse", (11, 10, 9), ["--dyn", "trt", "--omega", "1.6", "--magic",
                                                                     "0.25", "--ivel", "2", "--ivel-lid", "3",
                                                                     "--ulid", "0.05", "--local-rlb", "--steps", "80"]),
    "geo_channel_d3q19_lrlb_f64": ("d3q19_f64_nocse", (20, 12, 11), ["--dyn", "bgk", "--omega", "1.3", "--ivel", "3",
                                                                     "--poiseuille", "0.05", "--ipres", "4", "--rho",
                                                                     "0.99", "--bounceback", "2", "--bouzidi", "5",
                                                                     "--local-rlb", *RND, "--steps", "60"]),
    # two fluid dynamics in one block: ForcedBGK on material 1 and BGK on material 6 (periodic)
    "geo_two_dyn_d3q19_fbgk_bgk_f64": ("d3q19_f64_nocse", (12, 10, 9), ["--dyn", "fbgk", "--omega", "1.3", "--force",
                                                                        "1e-4", "2e-5", "0", "--periodic", "1", "1",
                                                                        "1", "--bgk-mat", "6", *RND, "--steps", "40"]),
    # two fluid dynamics of different kinds in one block: BGK on material 1, TRT on material 6;
    # and TRT on 1 with BGK on 6
    "geo_two_dyn_d3q19_bgk_trt_f64": ("d3q19_f64_nocse", (12, 10, 9), ["--dyn", "bgk", "--omega", "1.3", "--magic",
                                                                       "0.1", "--periodic", "1", "1", "1",
                                                                       "--trt-mat", "6", *RND, "--steps", "40"]),
    "geo_two_dyn_d2q9_trt_bgk_f64": ("d2q9_f64_nocse", (16, 14), ["--dyn", "trt", "--omega", "1.6", "--magic", "0.3",
                                                                  "--periodic", "1", "1", "--bgk-mat", "6", *RND,
                                                                  "--steps", "60"]),
    "geo_two_dyn_d2q9_fbgk_bgk_f64": ("d2q9_f64_nocse", (16, 14), ["--dyn", "fbgk", "--omega", "1.6", "--force",
                                                                   "1e-4", "-3e-5", "--periodic", "1", "1",
                                                                   "--bgk-mat", "6", *RND, "--steps", "60"]),
}
GEO_STEP = {"geo_step_d2q9_ivel_bgk_f64": (slice(8, None), slice(None, 5)),
            "geo_step_d3q19_ivel_bgk_f64": (slice(7, None), slice(None, 5), slice(6, None)),
            "geo_step_d3q27_ivel_trt_f64": (slice(6, None), slice(None, 5), slice(5, None)),
            "geo_step_d3q19_lvel_bgk_f64": (slice(7, None), slice(None, 5), slice(6, None)),
            "geo_step_d3q19_ivel_bgk_f32": (slice(7, None), slice(None, 5), slice(6, None)),
            "geo_step_d3q27_lrlb_trt_f64": (slice(6, None), slice(None, 5), slice(5, None))}
GEO_SPHERE = {"geo_channel_d3q27_trt_f64": (8, 7, 7, 3), "geo_channel_d3q27_trt_f32": (8, 7, 7, 3),
              "geo_channel_d3q19_bgk_rnd_f64": (6, 5, 6, 2.5), "geo_channel_d3q19_lvel_lpres_f64": (6, 5, 6, 2.5),
              "geo_channel_d3q19_lrlb_f64": (6, 5, 6, 2.5)}


def geo_material(name: str) -> np.ndarray:
    shape = GEO[name][1]
    if name in GEO_SPHERE:
        return geo_channel(shape, GEO_SPHERE[name])
    if "_two_dyn_" in name:
        return geo_two_dynamics(shape)
    if name in GEO_STEP:
        return geo_step(shape, GEO_STEP[name])
    return geo_box(shape)


STATS_EVERY = {"full_cavity_d2q9_bgk_128_f64": 100}


def select_stats(stats: np.ndarray, every: int) -> np.ndarray:
    """Every `every`-th row of per-step statistics, and the last row."""
    return np.vstack([stats[::every], stats[-1:]]) if every > 1 else stats


def generate(name: str) -> Path:
    if name in GEO:
        binary, shape, geo_args = GEO[name]
        case, args = "geo", ["--n", *map(str, shape), *geo_args]
    else:
        binary, case, args = CASES[name]
    exe = REF / f"lbref_{binary}"
    if not exe.exists():
        raise SystemExit(f"{exe} missing: build it with `make -C oracle ref`")
    with tempfile.TemporaryDirectory() as tmp:
        prefix = str(Path(tmp) / "c")
        if case == "geo":
            geo_material(name).tofile(prefix + ".in.mat")
            args = [*args, "--mat", prefix + ".in.mat"]
        subprocess.run([str(exe), case, *args, "--out", prefix], check=True, timeout=600, cwd=tmp,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        meta = json.loads(Path(prefix + ".json").read_text())
        dt = np.float64 if meta["bytes"] == 8 else np.float32
        q = meta["q"]
        n = int(np.prod(meta["ext"]))
        f0 = np.fromfile(prefix + ".f0.bin", dtype=dt).reshape(q, n)
        fS = np.fromfile(prefix + ".fS.bin", dtype=dt).reshape(q, n)
        mat = np.fromfile(prefix + ".mat.bin", dtype=np.int32)
        stats = np.loadtxt(prefix + ".stats.txt", ndmin=2)
        bnd = Path(prefix + ".bnd.bin")
        extra = {"bnd": np.fromfile(bnd, dtype=np.float64).reshape(-1, 8)} if bnd.exists() else {}
        vals = Path(prefix + ".vals.bin")
        if vals.exists():
            extra["vals"] = np.fromfile(vals, dtype=np.float64).reshape(-1, 4)
        bclass = Path(prefix + ".bclass.bin")
        if bclass.exists():
            extra["bclass"] = np.fromfile(bclass, dtype=np.int32).reshape(-1, 6)
        force = Path(prefix + ".force.txt")
        if force.exists():
            extra["force"] = np.loadtxt(force, ndmin=2)
    every = STATS_EVERY.get(name, 1)
    stats = select_stats(stats, every)
    meta["stats_every"] = every
    meta["binary"] = binary
    meta["args"] = [case, *[a for a in args if not a.endswith(".in.mat")]]
    out = HERE / f"{name}.npz"
    np.savez_compressed(out, f0=f0, fS=fS, mat=mat, stats=stats, meta=json.dumps(meta), **extra)
    return out


def main(argv: list[str]) -> int:
    names = argv or [*CASES, *GEO]
    for name in names:
        print(generate(name))
    return 0


if __name__ == "__main__":
    raise SystemExit(main(sys.argv[1:]))
