"""FP32-storage mode against the FP64 path (B200).

The mode stores ux, uy, uz, t, the predictor source terms and the Poisson
spectra in 4 bytes; p, psi, every coefficient and all arithmetic stay FP64.
It has no counterpart in the reference, so its oracle is the FP64 path, which
the parity tests pin to the reference. Tolerances: one FP32 rounding is
2^-24 = 6e-8 relative; the bounds below leave room for its growth over the
steps run and are stated per test.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from simpletcsolver_b200 import abi, ic
from simpletcsolver_b200.solver import Solver
from tests._helpers import rel_l2

pytestmark = pytest.mark.gpu

FIELDS = ("ux", "uy", "uz", "t")


def _run(lib, d0, case, storage, nsteps):
    s = Solver.from_ic(d0, case=case, lib=lib, storage=storage)
    try:
        assert s.storage == storage
        s.push()
        dts = s.run(nsteps)
        s.pull(abi.FIELDS)
        out = {n: s.field(n).copy() for n in FIELDS + ("p",)}
        out["diag"] = s.diagnostics()
        out["dts"] = np.array(dts)
        return out
    finally:
        s.release()


def test_push_pull_round_trip_is_fp32_rounding(lib, tmp_path):
    """push then pull returns every stored field rounded once to FP32 (bit
    exact, halos included) and p unchanged."""
    case = ic.taylor_couette(20, 16, 8, 3400.0)
    d0 = ic.write_ic(case, str(tmp_path / "ic"))
    s = Solver.from_ic(d0, case=case, lib=lib, storage=4)
    try:
        ref = {n: s.field(n).copy() for n in FIELDS + ("p",)}
        s.push()
        for n in FIELDS + ("p",):
            s.field(n)[...] = -7.0
        s.pull(abi.FIELDS)
        for n in FIELDS:
            np.testing.assert_array_equal(s.field(n), ref[n].astype(np.float32).astype(np.float64), err_msg=n)
        np.testing.assert_array_equal(s.field("p"), ref["p"])
    finally:
        s.release()


@pytest.mark.parametrize("name", ["tc", "tcexp", "planar", "tc_radial320"])
def test_short_runs_track_fp64(lib, name, tmp_path):
    """Five steps of each boundary/implicitness family (and of a radial line
    longer than the predict kernel's 256 field threads): velocity and scalar
    within 1e-5 relative L2 of the FP64 path, p within 1e-4, the same time
    steps to 1e-5 and divergence at the FP32 storage floor (below 1e-4)."""
    case = {"tc": ic.taylor_couette(32, 32, 16, 3400.0),
            "tcexp": ic.taylor_couette(20, 16, 8, 3400.0, implicit=(False, False, False)),
            "planar": ic.plane_couette(24, 16, 16, 2000.0),
            "tc_radial320": ic.taylor_couette(320, 16, 8, 1.0e4)}[name]
    d0 = ic.write_ic(case, str(tmp_path / "ic"))
    a = _run(lib, d0, case, 8, 5)
    b = _run(lib, d0, case, 4, 5)
    for n in FIELDS:
        assert rel_l2(b[n][1:-1, 1:-1], a[n][1:-1, 1:-1]) < 1e-5, n
    pa, pb = a["p"][1:-1, 1:-1], b["p"][1:-1, 1:-1]
    assert rel_l2(pb - pb.mean(), pa - pa.mean()) < 1e-4
    np.testing.assert_allclose(b["dts"], a["dts"], rtol=1e-5)
    assert b["diag"]["divmax"] < 1e-4


def test_taylor_couette_64x128x64_100_steps(lib, tmp_path):
    """The CPU-runnable Taylor-Couette workload, 100 steps: velocity within
    1e-4 relative L2 of FP64, inner-wall torque (the energy injection, the
    outer wall being at rest) and dissipation within 1e-5, divergence below
    1e-4."""
    case = ic.TC_SMALL
    d0 = ic.write_ic(case, str(tmp_path / "ic"))
    a = _run(lib, d0, case, 8, 100)
    b = _run(lib, d0, case, 4, 100)
    for n in FIELDS:
        assert rel_l2(b[n][1:-1, 1:-1], a[n][1:-1, 1:-1]) < 1e-4, n
    for k in ("injection_u", "dissipation_u"):
        assert abs(b["diag"][k] - a["diag"][k]) <= 1e-5 * abs(a["diag"][k]), k
    assert b["diag"]["divmax"] < 1e-4
    assert a["diag"]["divmax"] < 1e-12


def test_storage_selection_is_per_context(lib, tmp_path):
    """A context keeps the storage it was created with; the default for new
    contexts is restored by Solver.from_ic."""
    case = ic.taylor_couette(16, 16, 8, 3400.0)
    d0 = ic.write_ic(case, str(tmp_path / "ic"))
    s4 = Solver.from_ic(d0, case=case, lib=lib, storage=4)
    s8 = Solver.from_ic(d0, case=case, lib=lib)
    try:
        assert s4.storage == 4 and s8.storage == 8
        assert lib.tcgpu_get_storage(None) == 8
        s4.push(); s8.push()
        s4.run(2); s8.run(2)
        assert s4.storage == 4 and s8.storage == 8
    finally:
        s4.release(); s8.release()
