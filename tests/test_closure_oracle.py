"""CPU checks of the closure oracle (oracle/closure_ref.py): the restriction
keeps a divergence-free field divergence-free on the coarse grid, is exact
on fields constant along each coarse cell, and Adam's first step has the
closed form -lr sign(g)."""
from __future__ import annotations

import numpy as np

from oracle import closure_ref as cr
from oracle import tc_numpy as tn
from simpletcsolver_b200 import closure, ic
from tests._helpers import params_of


def _coarse_domain(case, tmp_path):
    dc = closure.write_coarse_ic(case, str(tmp_path / "coarse"))
    return tn.load_domain(dc)


def test_restriction_keeps_the_velocity_divergence_free(tmp_path):
    case = ic.taylor_couette(16, 16, 8, 3400.0)
    d0 = ic.write_ic(case, str(tmp_path / "fine"))
    d = tn.load_domain(d0)
    fl = tn.load_fluid(d, d0, case.Re, case.Pr, params_of(case))
    tn.integrate(d, fl, params_of(case))          # the projection leaves div u at round-off
    fine_div = np.abs(tn.divergence(d, fl.ux, fl.uy, fl.uz)).max()
    assert fine_div < 1e-12
    c = cr.restrict({"ux": fl.ux, "uy": fl.uy, "uz": fl.uz, "t": fl.t, "p": fl.p}, d)
    dcd = _coarse_domain(case, tmp_path)
    nx, ny, nz = dcd.nx, dcd.ny, dcd.nz
    ux = tn.full(dcd)
    uy = tn.full(dcd)
    uz = tn.full(dcd)
    ux[1:-1, 1:-1, 1:nx + 1] = c["ux"]
    uy[1:-1, 1:-1, 1:nx + 1] = c["uy"]
    uz[1:-1, 1:-1, 1:nx + 1] = c["uz"]
    tn.bc_ux(dcd, ux)
    for a in (ux, uy, uz):
        tn.halo_yz(a)
    assert np.abs(tn.divergence(dcd, ux, uy, uz)).max() < 1e-12


def test_restriction_of_piecewise_constant_fields_is_exact(tmp_path):
    case = ic.taylor_couette(16, 16, 8, 3400.0)
    d0 = ic.write_ic(case, str(tmp_path / "fine"))
    d = tn.load_domain(d0)
    rng = np.random.default_rng(0)
    vals = rng.standard_normal((2, 4, 4))            # one value per coarse cell (k, j, i)
    rep = np.repeat(np.repeat(np.repeat(vals, 4, 0), 4, 1), 4, 2)
    f = {n: tn.full(d) for n in ("ux", "uy", "uz", "t", "p")}
    for n in f:
        f[n][1:-1, 1:-1, 1:d.nx + 1] = rep
    c = cr.restrict(f, d)
    for n in ("uy", "uz", "t", "p"):
        np.testing.assert_allclose(c[n], vals, rtol=1e-14, atol=1e-14)
    np.testing.assert_allclose(c["ux"][:, :, 1:], vals[:, :, 1:], rtol=1e-14, atol=1e-14)
    assert np.all(c["ux"][:, :, 0] == 0.0)


def test_adam_first_step_closed_form():
    g = np.array([3.0, -0.5, 1e-3])
    p, _, _ = cr.adam(np.zeros(3), g, np.zeros(3), np.zeros(3), 1, lr=0.01)
    np.testing.assert_allclose(p, -0.01 * np.sign(g), rtol=1e-4)
