"""The numpy restatement (oracle/tc_numpy.py) pinned against the reference.

Golden fixtures were produced by the reference's own C sources compiled
against single-rank shims (tests/golden/make_golden.py); where that build is
present the oracle is also checked against it directly on fresh cases.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from oracle import tc_numpy as tn
from simpletcsolver_b200 import ic
from tests._helpers import (demean, have_ref, load_golden, oracle_from_golden, oracle_layout, params_of, rel_l2,
                            REF_DIR)


@pytest.mark.parametrize("name", ["tc", "tcexp", "planar"])
def test_oracle_matches_reference_golden(name):
    z, meta, case = load_golden(name)
    d, fl = oracle_from_golden(z, case)
    prm = params_of(case)
    time = 0.0
    for _ in range(meta["steps"]):
        dt = tn.integrate(d, fl, prm, gauge="pin")
        time += dt
    assert dt == pytest.approx(meta["dt_last"], rel=1e-13)
    assert time == pytest.approx(meta["time"], rel=1e-13)
    for n in ("ux", "uy", "uz", "t"):
        ref = oracle_layout(n, z["ref_" + n])
        assert rel_l2(getattr(fl, n)[1:-1, 1:-1, 1:], ref[1:-1, 1:-1, 1:]) < 1e-12, n
    # pressure carries an arbitrary additive constant in the reference (singular mode)
    assert rel_l2(demean(fl.p), demean(z["ref_p"])) < 1e-11


@pytest.mark.parametrize("name", ["tc", "planar"])
def test_oracle_logging_matches_reference_golden(name):
    z, meta, case = load_golden(name)
    d, fl = oracle_from_golden(z, case)
    prm = params_of(case)
    for _ in range(meta["steps"]):
        tn.integrate(d, fl, prm)
    got = tn.diagnostics(d, fl)
    logs = meta["logs"]
    assert got["divmax"] < 1e-12 and logs["divergence"][0] < 1e-12
    assert got["injection_u"] == pytest.approx(logs["injection"][0], rel=1e-9)
    assert got["injection_t"] == pytest.approx(logs["injection"][1], rel=1e-9)
    assert got["dissipation_u"] == pytest.approx(logs["dissipation"][0], rel=1e-9)
    assert got["dissipation_t"] == pytest.approx(logs["dissipation"][1], rel=1e-9)
    for q, key in enumerate(("energy_ux", "energy_uy", "energy_uz", "energy_t")):
        assert got[key] == pytest.approx(logs["total_energy"][q], rel=1e-12)


@pytest.mark.parametrize("key", ["nr", "nc", "pr", "pc"])
def test_oracle_tdm_bit_exact_with_reference(key):
    """gtsv / periodic Sherman-Morrison restatement vs reference tdm.solve()."""
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "tdm.npz"))
    l, c, u, q, x = z[f"{key}_l"], z[f"{key}_c"], z[f"{key}_u"], z[f"{key}_q"], z[f"{key}_x"]
    data = q.copy()
    if data.ndim == 3:
        data = data[..., 0] + 1j * data[..., 1]
    rhs = np.moveaxis(data, 1, 0).copy()
    if key[0] == "p":
        tn.tdm_periodic(l, c, u, rhs)
    else:
        tn.gtsv(l, c, u, rhs)
    got = np.moveaxis(rhs, 0, 1)
    if x.ndim == 3:
        got = np.stack([got.real, got.imag], axis=-1)
    np.testing.assert_array_equal(got, x)


@pytest.mark.skipif(not have_ref("tc"), reason="reference build oracle/_ref absent")
@pytest.mark.parametrize("build,nx,ny,nz", [("tc", 10, 16, 8), ("tc", 12, 64, 16), ("tcexp", 12, 16, 8),
                                             ("planar", 10, 8, 16),
                                             # lengths that are not powers of two (the shim's direct DFT)
                                             ("tc", 10, 24, 12), ("planar", 10, 12, 20)])
def test_oracle_matches_reference_fresh_case(build, nx, ny, nz, tmp_path):
    if build == "planar":
        case = ic.plane_couette(nx, ny, nz, 2000.0, seed=7)
    else:
        case = ic.taylor_couette(nx, ny, nz, 3400.0, seed=7, implicit=(build == "tc", False, False))
    d0 = ic.write_ic(case, str(tmp_path / "ic"))
    out = str(tmp_path / "out")
    env = dict(os.environ, **ic.case_env(case))
    subprocess.run([os.path.join(REF_DIR, f"tcref_{build}"), d0, "0", "6", out], env=env, check=True,
                   capture_output=True)
    prm = params_of(case)
    d = tn.load_domain(d0)
    fl = tn.load_fluid(d, d0, case.Re, case.Pr, prm)
    for _ in range(6):
        tn.integrate(d, fl, prm)
    for n in ("ux", "uy", "uz", "t"):
        ref = tn.from_npy(d, n, np.load(os.path.join(out, n + ".npy")))
        assert rel_l2(tn.V(d, getattr(fl, n), 1, nx), tn.V(d, ref, 1, nx)) < 1e-12, n


def test_fft_shim_matches_numpy():
    """The shim FFT used by the reference build follows FFTW conventions."""
    src = os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle", "shim")
    prog = r'''
#include <stdio.h>
#include <complex.h>
#include "fftw3.h"
int main(void){
  enum {N = 16, M = 12};
  double in[N]; fftw_complex out[N/2+1]; double back[N];
  fftw_complex zin[M], zout[M];
  for(int i=0;i<N;i++) in[i] = (i*7%5) - 1.5 + 0.1*i;
  for(int i=0;i<M;i++) zin[i] = (i%3) + I*(i*0.25 - 1.);
  int n = N, m = M;
  fftw_plan p = fftw_plan_many_dft_r2c(1, &n, 1, in, NULL, 1, N, out, NULL, 1, N/2+1, FFTW_MEASURE);
  fftw_execute(p);
  fftw_plan q = fftw_plan_many_dft_c2r(1, &n, 1, out, NULL, 1, N/2+1, back, NULL, 1, N, FFTW_MEASURE);
  fftw_execute(q);
  fftw_plan r = fftw_plan_many_dft(1, &m, 1, zin, NULL, 1, M, zout, NULL, 1, M, FFTW_FORWARD, FFTW_MEASURE);
  fftw_execute(r);
  for(int i=0;i<N/2+1;i++) printf("%.17e %.17e\n", creal(out[i]), cimag(out[i]));
  for(int i=0;i<N;i++) printf("%.17e\n", back[i]);
  for(int i=0;i<M;i++) printf("%.17e %.17e\n", creal(zout[i]), cimag(zout[i]));
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as td:
        cfile = os.path.join(td, "t.c")
        open(cfile, "w").write(prog)
        exe = os.path.join(td, "t")
        subprocess.run(["gcc", "-std=c99", "-O2", "-I", src, cfile, os.path.join(src, "fftw_shim.c"), "-lm", "-o", exe],
                       check=True)
        vals = np.array([float(v) for v in subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()])
    N, M = 16, 12
    x = np.array([(i * 7 % 5) - 1.5 + 0.1 * i for i in range(N)])
    z = np.array([(i % 3) + 1j * (i * 0.25 - 1.0) for i in range(M)])
    r2c = vals[:2 * (N // 2 + 1)].reshape(-1, 2)
    np.testing.assert_allclose(r2c[:, 0] + 1j * r2c[:, 1], np.fft.rfft(x), rtol=0, atol=1e-12)
    back = vals[2 * (N // 2 + 1):2 * (N // 2 + 1) + N]
    np.testing.assert_allclose(back, N * x, rtol=0, atol=1e-11)
    c2c = vals[2 * (N // 2 + 1) + N:].reshape(-1, 2)
    np.testing.assert_allclose(c2c[:, 0] + 1j * c2c[:, 1], np.fft.fft(z), rtol=0, atol=1e-12)
