"""The initial field generated on the device (tcgpu_fluid_init_generated).

The seeded numpy generator (simpletcsolver_b200/ic.py) writes NPY files that
both the reference and this library read; at 256x1024x512 that is 1.1 GB per
field. The device generator makes the same kind of field in place: the laminar
profile plus uniform noise, with the wall values and periodic images of
fluid_init. Its noise is a function of (seed, field, cell), so it is
reproducible but not numpy's sequence; these tests check the field's
definition, not equality with ic.py.
"""
import numpy as np
import pytest

from simpletcsolver_b200 import ic
from simpletcsolver_b200.solver import Solver

pytestmark = pytest.mark.gpu


def fields(s):
    return {n: s.field(n).copy() for n in ("ux", "uy", "uz", "p", "t")}


@pytest.mark.parametrize("curved", [True, False])
def test_generated_field_follows_its_definition(lib, tmp_path, curved):
    case = (ic.taylor_couette(32, 64, 16, 3400.0, seed=7) if curved
            else ic.plane_couette(24, 32, 16, 2000.0, seed=7))
    s = Solver.from_case(case, str(tmp_path / "a"), lib=lib)
    try:
        f = fields(s)
        xf, xc = ic.radial_grid(case)
        ri, ro = xf[0], xf[-1]
        if curved:
            A = (case.uy_xp * ro - case.uy_xm * ri) / (ro * ro - ri * ri)
            B = (case.uy_xm - A * ri) * ri
            prof = A * xc + B / xc
        else:
            prof = case.uy_xm + (case.uy_xp - case.uy_xm) * (xc - ri) / case.lx
        tprof = case.t_xm + (case.t_xp - case.t_xm) * (xc - ri) / case.lx
        a = case.noise_u
        dev = f["uy"][1:-1, 1:-1, 1:-1] - prof[None, None, 1:-1]
        assert np.all(dev >= -a) and np.all(dev < a) and abs(dev.mean()) < 0.02 * a
        assert abs(dev.std() - a / np.sqrt(3.0)) < 0.02 * a           # uniform on [-a, a)
        for n in ("uz",):
            v = f[n][1:-1, 1:-1, 1:-1]
            assert np.all(np.abs(v) <= a) and abs(v.mean()) < 0.02 * a
        ux = f["ux"][1:-1, 1:-1]
        assert not ux[:, :, 0].any() and not ux[:, :, -1].any()        # impermeable walls
        assert np.all(np.abs(ux[:, :, 1:-1]) <= a) and ux[:, :, 1:-1].std() > 0.5 * a / np.sqrt(3.0)
        t = f["t"][1:-1, 1:-1, 1:-1] - tprof[None, None, 1:-1]
        at = case.noise_t
        assert np.all(np.abs(t) <= at + 1e-14)      # the profile itself agrees to round-off
        assert not f["p"].any()
        # walls and periodic images as fluid_init leaves them
        assert np.all(f["uy"][:, :, 0] == case.uy_xm) and np.all(f["uy"][:, :, -1] == case.uy_xp)
        assert np.array_equal(f["uy"][1:-1, 0], f["uy"][1:-1, -2])
        assert np.array_equal(f["uy"][0], f["uy"][-2])
        # the same seed gives the same field, another seed another one
        r = Solver.from_case(case, str(tmp_path / "b"), lib=lib)
        g = fields(r)
        r.release()
        for n in f:
            np.testing.assert_array_equal(f[n], g[n], err_msg=n)
        other = ic.Case(**{**case.__dict__, "seed": 8})
        r = Solver.from_case(other, str(tmp_path / "c"), lib=lib)
        assert not np.array_equal(fields(r)["uy"], f["uy"])
        r.release()
        # and it steps: divergence at round-off after one step
        s.integrate()
        assert s.diagnostics()["divmax"] < 1e-12
    finally:
        s.release()


def test_generated_field_in_fp32_storage(lib, tmp_path):
    """The same field with 4-byte storage: one FP32 rounding of the FP64 field
    (p stays FP64 and zero)."""
    case = ic.taylor_couette(24, 32, 16, 3400.0, seed=11)
    a = Solver.from_case(case, str(tmp_path / "a"), lib=lib)
    b = Solver.from_case(case, str(tmp_path / "b"), lib=lib, storage=4)
    try:
        assert b.storage == 4
        fa, fb = fields(a), fields(b)
        for n in ("ux", "uy", "uz", "t"):
            np.testing.assert_array_equal(fb[n], fa[n].astype(np.float32).astype(np.float64), err_msg=n)
        assert not fb["p"].any()
        b.integrate()
        assert b.diagnostics()["divmax"] < 1e-4
    finally:
        a.release()
        b.release()


def test_generated_field_at_the_headline_grid(lib, tmp_path):
    """256x1024x512 without any field file: generated, stepped resident, and
    divergence-free to round-off after the first step."""
    case = ic.TC_LARGE
    s = Solver.from_case(case, str(tmp_path / "ic"), lib=lib)
    try:
        s.push()
        dts = s.run(2)
        assert np.all(dts > 0)
        xf = ic.radial_grid(case)[0]
        assert s.diagnostics()["divmax"] < 1e-13 * 1.1 / float(np.min(np.diff(xf)))
    finally:
        s.release()
