"""Seeded initial-condition generator: the reference's NPY schema
(initial_condition/main.py:46-103) and the laminar profiles."""
import os
import subprocess

import numpy as np
import pytest

from simpletcsolver_b200 import ic
from tests._helpers import REF_DIR, have_ref


def test_schema_and_profiles(tmp_path):
    case = ic.taylor_couette(16, 8, 4, 3400.0, noise_u=0.0)
    d = ic.write_ic(case, str(tmp_path))
    shapes = {"ux": (4, 8, 17), "uy": (4, 8, 18), "uz": (4, 8, 18), "p": (4, 8, 18), "t": (4, 8, 18),
              "xf": (17,), "xc": (18,), "glsizes": (3,), "lengths": (3,), "is_curved": (), "step": (), "time": ()}
    dtypes = {"glsizes": np.uint64, "step": np.uint64, "is_curved": np.bool_}
    for n, s in shapes.items():
        a = np.load(os.path.join(d, n + ".npy"))
        assert a.shape == s, n
        assert a.dtype == dtypes.get(n, np.float64), n
    xf = np.load(os.path.join(d, "xf.npy"))
    xc = np.load(os.path.join(d, "xc.npy"))
    assert xf[0] == 1.0 and xf[-1] == pytest.approx(1.4)
    assert xc[0] == xf[0] and xc[-1] == xf[-1]
    assert np.all(np.diff(xf) > 0)
    uy = np.load(os.path.join(d, "uy.npy"))
    # circular Couette: uy(ri) = 1, uy(ro) = 0, A r + B / r in between
    assert uy[0, 0, 0] == pytest.approx(1.0) and abs(uy[0, 0, -1]) < 1e-12
    ri, ro = 1.0, 1.4
    a = -ri * ri / (ro * ro - ri * ri)
    b = (1.0 - a * ri) * ri
    np.testing.assert_allclose(uy[0, 0], a * xc + b / xc, rtol=1e-13)


def test_seeded_noise_is_reproducible(tmp_path):
    c = ic.taylor_couette(8, 8, 4, 3400.0, seed=3)
    f1 = ic.initial_fields(c)
    f2 = ic.initial_fields(c)
    for n in f1:
        np.testing.assert_array_equal(f1[n], f2[n])
    assert np.abs(f1["ux"]).max() <= 0.05 and np.abs(f1["ux"]).max() > 0.01


@pytest.mark.skipif(not have_ref("planar"), reason="reference build oracle/_ref absent")
def test_reference_loads_generated_ic(tmp_path):
    case = ic.plane_couette(8, 8, 8, 2000.0)
    d = ic.write_ic(case, str(tmp_path / "ic"))
    env = dict(os.environ, **ic.case_env(case))
    r = subprocess.run([os.path.join(REF_DIR, "tcref_planar"), d, "0", "1"], env=env, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert '"cells": 512' in r.stdout
