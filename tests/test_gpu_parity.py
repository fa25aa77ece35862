"""GPU parity: libtcgpu.so through its C ABI against the oracle and the
reference's own results.

Tolerances (FP64 throughout): fields within 1e-12 of the oracle per stage
(relative to the field's magnitude), 1e-12 relative L2 against the golden
reference runs and 1e-10 relative L2 after 100 steps of the 64x128x64
Taylor-Couette case; pressure and potential are compared after removing their
mean because the reference leaves the additive constant of the singular
Poisson mode to round-off.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from oracle import tc_numpy as tn
from simpletcsolver_b200 import abi, ic
from simpletcsolver_b200.solver import Solver, SolverError
from tests._helpers import (REF_DIR, demean, have_ref, load_golden, oracle_from_golden, oracle_layout, params_of,
                            rel_l2, write_ic_from_golden)

pytestmark = pytest.mark.gpu

CASES = {
    "tc": ic.taylor_couette(16, 32, 16, 3400.0),
    "tcexp": ic.taylor_couette(20, 16, 8, 3400.0, implicit=(False, False, False)),
    "planar": ic.plane_couette(12, 16, 8, 2000.0),
    # y and z lines of 64 and 128 points: the warp-per-line periodic solves
    "planar_lines": ic.plane_couette(12, 64, 128, 2000.0),
    # 64 radial points: the Poisson radial solves by warps over tiles of lines
    "tc_radial64": ic.taylor_couette(64, 16, 8, 3400.0),
    # 128 and 256 radial points: predict kernels of 4 and 8 warps per line, Poisson solves with 4 and 8 points per lane
    "tc_radial128": ic.taylor_couette(128, 16, 8, 1.0e4),
    "tc_radial256": ic.taylor_couette(256, 16, 8, 1.0e4),
    # y lines of 1024 and 512 points: y transforms whose lines are two warps and
    # one warp (barriers per line), 12 radial points so that the second CTA of
    # 8 radial indices has idle ones
    "tc_lines_y1024": ic.taylor_couette(12, 1024, 8, 3400.0),
    "tc_lines_y512": ic.taylor_couette(12, 512, 16, 3400.0),
    # lengths that are not powers of two: direct transforms in y and z, plane
    # chunks that divide nz (96 = 3 x 32 points in y, 48 and 36 in z)
    "tc_y96_z48": ic.taylor_couette(16, 96, 48, 3400.0),
    # radial lines longer than the predict kernel's 256 field threads: tiles of
    # 256 radial indices, then the line solves (x; and y, z in the planar case)
    "tc_radial384": ic.taylor_couette(384, 16, 8, 1.0e4),
    "tc_radial512": ic.taylor_couette(512, 16, 8, 1.0e4),
    "planar_radial320": ic.plane_couette(320, 16, 8, 2000.0),
    "planar_y48_z36": ic.plane_couette(12, 48, 36, 2000.0),
}

# Tolerance multipliers. With 512 and 1024 azimuthal points the spacing is
# r dy = 6e-4 to 1.2e-3, so the y advection fluxes entering the source terms are
# about 1e4 times larger than the terms themselves (|src| <= 0.12): rounding of
# the addends alone reaches 2e-12 of the result.
TOL_SCALE = {"tc_lines_y1024": 10.0, "tc_lines_y512": 10.0}


def close(gpu, orc, name, tol=1e-12):
    if name == "ux":
        orc = orc[:, :, 1:]
    scale = max(np.abs(orc).max(), 1e-300)
    err = np.abs(gpu - orc).max() / scale
    assert err < tol, f"{name}: max error {err:.3e} relative to {scale:.3e}"


@pytest.mark.parametrize("name", list(CASES))
def test_every_stage_matches_oracle(lib, name, tmp_path):
    case = CASES[name]
    f = TOL_SCALE.get(name, 1.0)
    d0 = ic.write_ic(case, str(tmp_path / "ic"))
    prm = params_of(case)
    d = tn.load_domain(d0)
    fl = tn.load_fluid(d, d0, case.Re, case.Pr, prm)
    s = Solver.from_ic(d0, case=case, lib=lib, coherence=abi.SYNC_SRCS)
    try:
        for n in ("ux", "uy", "uz", "p", "t"):
            close(s.field(n), getattr(fl, n), n, tol=0.0 + 1e-300)
        dt = tn.decide_dt(d, fl, prm)
        assert s.decide_dt() == dt          # same arithmetic: bit-identical
        for rk in range(3):
            tn.predict_field(d, rk, dt, fl, prm)
            s.predict(rk, dt)
            for n in ("ux", "uy", "uz", "t"):
                close(s.field(n), getattr(fl, n), n, tol=1e-12 * f)
            for v in ("ux", "uy", "uz", "t"):
                o = fl.src[v][0]
                assert np.abs(s.src(v, 0) - o).max() <= 1e-12 * f * max(np.abs(o).max(), 1e-300), f"srcA {v} rk{rk}"
            tn.compute_potential(d, rk, dt, fl)
            s.compute_potential(rk, dt)
            close(s.field("psi"), fl.psi, "psi", tol=1e-11 * f)
            tn.correct_velocity(d, rk, dt, fl, prm)
            s.correct_velocity(rk, dt)
            for n in ("ux", "uy", "uz"):
                close(s.field(n), getattr(fl, n), n, tol=1e-12 * f)
            tn.update_pressure(d, rk, dt, fl, prm)
            s.update_pressure(rk, dt)
            close(s.field("p"), fl.p, "p", tol=1e-11 * f)
    finally:
        s.release()


@pytest.mark.parametrize("name", ["tc", "tcexp", "planar"])
def test_integrate_matches_reference_golden(lib, name, tmp_path):
    z, meta, case = load_golden(name)
    d0 = write_ic_from_golden(z, str(tmp_path / "ic"))
    s = Solver.from_ic(d0, case=case, lib=lib)
    try:
        time = 0.0
        for _ in range(meta["steps"]):
            dt = s.integrate()
            time += dt
        assert dt == pytest.approx(meta["dt_last"], rel=1e-13)
        assert time == pytest.approx(meta["time"], rel=1e-13)
        for n in ("ux", "uy", "uz", "t"):
            assert rel_l2(s.field(n)[1:-1, 1:-1], z["ref_" + n][1:-1, 1:-1]) < 1e-12, n
        assert rel_l2(demean(s.field("p")), demean(z["ref_p"])) < 1e-11
        logs = meta["logs"]
        got = s.diagnostics()
        assert got["divmax"] < 1e-12
        assert got["injection_u"] == pytest.approx(logs["injection"][0], rel=1e-9)
        assert got["injection_t"] == pytest.approx(logs["injection"][1], rel=1e-9)
        assert got["dissipation_u"] == pytest.approx(logs["dissipation"][0], rel=1e-9)
        assert got["dissipation_t"] == pytest.approx(logs["dissipation"][1], rel=1e-9)
        for q, key in enumerate(("energy_ux", "energy_uy", "energy_uz", "energy_t")):
            assert got[key] == pytest.approx(logs["total_energy"][q], rel=1e-11)
    finally:
        s.release()


@pytest.mark.skipif(not have_ref("tc"), reason="reference build oracle/_ref absent")
def test_100_steps_taylor_couette_64x128x64(lib, tmp_path):
    """The CPU-runnable Taylor-Couette workload: 100 steps on the GPU against
    100 steps of the reference, every field within 1e-10 relative L2."""
    case = ic.TC_SMALL
    d0 = ic.write_ic(case, str(tmp_path / "ic"))
    out = str(tmp_path / "ref")
    env = dict(os.environ, **ic.case_env(case))
    ref = subprocess.Popen([os.path.join(REF_DIR, "tcref_tc"), d0, "0", "100", out], env=env,
                           stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
    s = Solver.from_ic(d0, case=case, lib=lib)
    try:
        s.push()
        s.run(100)
        s.pull(abi.FIELDS)
        diag = s.diagnostics()
        stdout, stderr = ref.communicate(timeout=1800)
        assert ref.returncode == 0, stderr
        for n in ("ux", "uy", "uz", "t"):
            r = np.load(os.path.join(out, n + ".npy"))
            assert rel_l2(s.field(n)[1:-1, 1:-1], r) < 1e-10, n
        rp = np.load(os.path.join(out, "p.npy"))
        gp = s.field("p")[1:-1, 1:-1]
        assert rel_l2(gp - gp[:, :, 1:-1].mean(), rp - rp[:, :, 1:-1].mean()) < 1e-10
        assert diag["divmax"] < 1e-12
    finally:
        s.release()


@pytest.mark.parametrize("key", ["nr", "nc", "pr", "pc"])
def test_tdm_bit_exact_with_reference(lib, key):
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "tdm.npz"))
    l, c, u, q, x = z[f"{key}_l"], z[f"{key}_c"], z[f"{key}_u"], z[f"{key}_q"], z[f"{key}_x"]
    tdm = abi.tdm_vtable(lib)
    n, nrhs = l.shape[0], q.shape[0]
    info = abi.TdmInfoP()
    assert tdm.construct(n, nrhs, key[0] == "p", key[1] == "c", C.byref(info)) == 0
    ptr = abi.c_double_p()
    for nm, v, getter in (("l", l, tdm.get_l), ("c", c, tdm.get_c), ("u", u, tdm.get_u)):
        getter(info, C.byref(ptr))
        np.ctypeslib.as_array(ptr, shape=(n,))[:] = v
    data = np.ascontiguousarray(q.copy())
    assert tdm.solve(info, data.ctypes.data_as(C.c_void_p)) == 0
    np.testing.assert_array_equal(data, x)
    # device-resident right-hand sides are solved in place
    import torch
    dq = torch.from_numpy(np.ascontiguousarray(q.copy())).cuda()
    assert tdm.solve(info, C.c_void_p(dq.data_ptr())) == 0
    np.testing.assert_array_equal(dq.cpu().numpy(), x)
    assert tdm.destruct(info) == 0


def test_boundary_entry_points_match_oracle(lib, tmp_path):
    case = ic.taylor_couette(12, 8, 8, 3400.0)
    d0 = ic.write_ic(case, str(tmp_path / "ic"))
    # the wall values are the library's parameters, which earlier tests may have changed
    from simpletcsolver_b200.solver import params_of as solver_params
    assert lib.tcgpu_set_params(C.byref(solver_params(case))) == 0
    d = abi.DomainT()
    assert lib.domain_init(d0.encode(), C.byref(d)) == 0
    od = tn.load_domain(d0)
    prm = tn.Params()
    rng = np.random.default_rng(5)
    for name, fn in (("ux", tn.bc_ux), ("uy", lambda dd, a: tn.bc_uy(dd, a, prm)), ("uz", tn.bc_uz),
                     ("p", tn.bc_p), ("psi", tn.bc_psi), ("t", lambda dd, a: tn.bc_t(dd, a, prm))):
        row = case.nx + 1 if name == "ux" else case.nx + 2
        host = rng.standard_normal((case.nz + 2, case.ny + 2, row))
        arr = abi.ArrayT(8, None, host.nbytes, host.ctypes.data)
        expect = oracle_layout(name, host.copy())
        fn(od, expect)
        assert getattr(lib, f"fluid_update_boundaries_{name}")(C.byref(d), C.byref(arr)) == 0
        np.testing.assert_array_equal(host, expect[:, :, 1:] if name == "ux" else expect, err_msg=name)


def test_coherent_and_resident_paths_agree(lib, tmp_path):
    case = ic.taylor_couette(16, 16, 8, 3400.0)
    d0 = ic.write_ic(case, str(tmp_path / "ic"))
    a = Solver.from_ic(d0, case=case, lib=lib)
    b = Solver.from_ic(d0, case=case, lib=lib)
    try:
        dts_a = [a.integrate() for _ in range(4)]
        b.push()
        dts_b = b.run(4)
        b.pull()
        assert dts_a == list(dts_b)
        for n in ("ux", "uy", "uz", "p", "t", "psi"):
            np.testing.assert_array_equal(a.field(n), b.field(n), err_msg=n)
    finally:
        a.release()
        b.release()


def test_tensors_follow_reference_semantics(lib, tmp_path):
    """With TCGPU_SYNC_TENSORS the host tensors after a predict are those of
    the predict's input fields (src/fluid/predict/main.c:56-82)."""
    case = CASES["tc"]
    d0 = ic.write_ic(case, str(tmp_path / "ic"))
    prm = params_of(case)
    d = tn.load_domain(d0)
    fl = tn.load_fluid(d, d0, case.Re, case.Pr, prm)
    s = Solver.from_ic(d0, case=case, lib=lib, coherence=abi.SYNC_TENSORS)
    try:
        dt = s.decide_dt()
        tn.predict_field(d, 0, dt, fl, prm)
        s.predict(0, dt)
        for name, a in fl.tensors.items():
            g = s.tensor(name)
            face = name in ("lxy", "lxz", "lyx0", "lyx1", "lzx")
            o = a[:, :, 1:case.nx + 2] if face else a[:, :, 1:case.nx + 1]
            assert np.abs(g - o).max() <= 1e-12 * max(np.abs(o).max(), 1e-300), name
    finally:
        s.release()


def test_save_and_restart_in_reference_layout(lib, tmp_path):
    case = CASES["tc"]
    d0 = ic.write_ic(case, str(tmp_path / "ic"))
    s = Solver.from_ic(d0, case=case, lib=lib)
    try:
        t = sum(s.integrate() for _ in range(3))
        out = str(tmp_path / "save")
        s.save(out, step=3, time=t)
        r = Solver.from_ic(out, case=case, lib=lib)
        for n in ("ux", "uy", "uz", "p", "t"):
            np.testing.assert_array_equal(r.field(n), s.field(n), err_msg=n)
        assert int(np.load(os.path.join(out, "step.npy"))) == 3
        # the restart continues exactly like the uninterrupted run
        assert r.integrate() == s.integrate()
        np.testing.assert_array_equal(r.field("uy"), s.field("uy"))
        r.release()
    finally:
        s.release()


def test_laminar_couette_stays_axisymmetric(lib, tmp_path):
    """Circular Couette flow without noise: no radial or axial velocity appears
    and the azimuthal velocity stays independent of y and z."""
    case = ic.taylor_couette(24, 16, 8, 3400.0, noise_u=0.0)
    d0 = ic.write_ic(case, str(tmp_path / "ic"))
    s = Solver.from_ic(d0, case=case, lib=lib)
    try:
        s.push()
        s.run(20)
        s.pull()
        assert np.abs(s.field("ux")).max() < 1e-13
        assert np.abs(s.field("uz")).max() < 1e-13
        uy = s.field("uy")[1:-1, 1:-1]
        assert np.abs(uy - uy[:1, :1]).max() < 1e-13
        assert s.diagnostics()["divmax"] < 1e-13
    finally:
        s.release()


def test_nonfinite_field_is_reported_not_propagated(lib, tmp_path):
    """Failure detection without a device fault: a NaN in the host field makes
    the CFL reduction raise its status bit and integrate() return non-zero."""
    case = CASES["tc"]
    d0 = ic.write_ic(case, str(tmp_path / "ic"))
    s = Solver.from_ic(d0, case=case, lib=lib)
    try:
        s.field("uy")[3, 4, 5] = np.nan
        with pytest.raises(SolverError, match="non-finite"):
            s.integrate()
        # the context stays usable once the field is repaired
        s.field("uy")[3, 4, 5] = 0.5
        assert s.integrate() > 0.0
    finally:
        s.release()


def test_headline_grid_step_properties(lib, tmp_path):
    """256x1024x512 at Re=1e4: a few steps keep the velocity divergence-free to
    round-off and the budgets finite (size-independent properties)."""
    case = ic.TC_LARGE
    d0 = ic.write_ic(case, str(tmp_path / "ic"))
    s = Solver.from_ic(d0, case=case, lib=lib)
    try:
        s.push()
        dts = s.run(3)
        assert np.all(dts > 0) and np.all(np.isfinite(dts))
        diag = s.diagnostics()
        assert all(np.isfinite(v) for v in diag.values())
        # divergence at round-off of the largest velocity gradient
        s.pull(abi.UX)
        hmin = float(np.min(np.load(os.path.join(d0, "xf.npy"))[1:] - np.load(os.path.join(d0, "xf.npy"))[:-1]))
        assert diag["divmax"] < 1e-13 * 1.1 / hmin
    finally:
        s.release()
