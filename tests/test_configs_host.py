"""Host-side parts of the benchmark configurations (no GPU): the seeded sphere packing of the
porous medium and the command line of openlb_b200.configs."""
import subprocess
import sys

import numpy as np

from openlb_b200 import configs


def test_sphere_packing_is_seeded_and_reaches_its_porosity_range():
    a = configs.porous_spheres(64, seed=3)
    b = configs.porous_spheres(64, seed=3)
    c = configs.porous_spheres(64, seed=4)
    assert a.dtype == bool and a.shape == (64, 64, 64)
    assert np.array_equal(a, b)  # the same seed gives the same medium
    assert not np.array_equal(a, c)
    assert 0.595 < 1 - a.mean() <= 0.6  # the addition stops once the solid reaches 0.4


def test_spheres_wrap_across_the_periodic_faces():
    s = configs.porous_spheres(40, seed=1)
    # solid on a face continues on the opposite face for some sphere (periodic placement)
    assert (s[0] & s[-1]).any() or (s[:, 0] & s[:, -1]).any() or (s[:, :, 0] & s[:, :, -1]).any()


def test_command_line_help():
    out = subprocess.run([sys.executable, "-m", "openlb_b200.configs", "--help"], capture_output=True, text=True,
                         timeout=120)
    assert out.returncode == 0 and "channel" in out.stdout and "porous" in out.stdout
