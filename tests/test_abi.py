"""C-ABI boundary checks that need no GPU: exports, struct layout against the
reference's own headers and library, NPY start-up / save, error returns."""
import ctypes as C
import os
import subprocess
import tempfile

import numpy as np
import pytest

from oracle import tc_numpy as tn
from simpletcsolver_b200 import abi, ic
from tests._helpers import REF_DIR, have_ref


def test_exports_every_declared_symbol(lib):
    names = abi.declared_symbols()
    assert "integrate" in names and "tdm" in names and "fluid_predict_field" in names
    out = subprocess.run(["nm", "-D", "--defined-only", abi.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [n for n in names if n not in exported]
    assert not missing, missing


def test_every_declared_function_has_a_binding():
    """Every function include/tcgpu.h declares has a ctypes signature with the
    header's number of parameters."""
    fns = abi.declared_functions()
    assert {"integrate", "tcgpu_run_timed", "tcgpu_tdm_solve_noalloc", "tcgpu_nn_conv3"} <= set(fns)
    assert set(fns) <= set(abi.declared_symbols())
    sigs = {**abi._SIGS, **abi._EXT_SIGS}
    assert sorted(set(fns) - set(sigs)) == []
    wrong = {n: (fns[n], len(sigs[n][1])) for n in fns if len(sigs[n][1]) != fns[n]}
    assert wrong == {}


def test_struct_layout_matches_header(tmp_path):
    prog = r'''
#include <stdio.h>
#include <stddef.h>
#include "tcgpu.h"
int main(void){
  printf("%zu %zu %zu %zu\n", sizeof(array_t), sizeof(domain_t), sizeof(fluid_t), sizeof(tcgpu_params_t));
  printf("%zu %zu %zu %zu\n", offsetof(domain_t, glsizes), offsetof(domain_t, lengths), offsetof(domain_t, xf), offsetof(domain_t, hz));
  printf("%zu %zu %zu %zu\n", offsetof(fluid_t, srcux), offsetof(fluid_t, lxx), offsetof(fluid_t, lzz), offsetof(fluid_t, Re));
  return 0;
}
'''
    c = tmp_path / "l.c"
    c.write_text(prog)
    exe = tmp_path / "l"
    inc = os.path.join(os.path.dirname(abi.HEADER))
    subprocess.run(["gcc", "-std=c99", "-I", inc, str(c), "-o", str(exe)], check=True)
    v = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert v[:4] == [C.sizeof(abi.ArrayT), C.sizeof(abi.DomainT), C.sizeof(abi.FluidT), C.sizeof(abi.ParamsT)]
    assert v[4:8] == [abi.DomainT.glsizes.offset, abi.DomainT.lengths.offset, abi.DomainT.xf.offset, abi.DomainT.hz.offset]
    assert v[8:12] == [abi.FluidT.srcux.offset, abi.FluidT.lxx.offset, abi.FluidT.lzz.offset, abi.FluidT.Re.offset]


@pytest.mark.skipif(not have_ref("tc"), reason="reference build oracle/_ref absent")
def test_domain_init_matches_reference(lib, tmp_path):
    """The reference's domain_init fills the same struct; metrics are bit-identical."""
    case = ic.taylor_couette(12, 16, 8, 3400.0)
    d0 = ic.write_ic(case, str(tmp_path / "ic"))
    code = r'''
import ctypes as C, sys, numpy as np
sys.path.insert(0, %r)
from simpletcsolver_b200 import abi
ref = abi.bind_reference_api(C.CDLL(%r))
d = abi.DomainT()
assert ref.domain_init(%r, C.byref(d)) == 0
nx = d.glsizes[0]
out = {k: np.ctypeslib.as_array(getattr(d, k), shape=(nx + (1 if k in ("xf","hxxf","hyxf","jdxf") else 2),)).copy()
       for k in ("xf","xc","hxxf","hxxc","hyxf","hyxc","jdxf","jdxc")}
out["hz"] = np.array(d.hz); out["glsizes"] = np.array(list(d.glsizes)); out["mysizes"] = np.array(list(d.mysizes))
np.savez(%r, **out)
''' % (os.path.dirname(os.path.dirname(abi.__file__)), os.path.join(REF_DIR, "libtcref_tc.so"), d0.encode(),
       str(tmp_path / "ref.npz"))
    subprocess.run(["python", "-c", code], check=True, capture_output=True)
    ref = np.load(tmp_path / "ref.npz")
    d = abi.DomainT()
    assert lib.domain_init(d0.encode(), C.byref(d)) == 0
    nx = d.glsizes[0]
    for k in ("xf", "xc", "hxxf", "hxxc", "hyxf", "hyxc", "jdxf", "jdxc"):
        n = nx + (1 if k in ("xf", "hxxf", "hyxf", "jdxf") else 2)
        np.testing.assert_array_equal(np.ctypeslib.as_array(getattr(d, k), shape=(n,)), ref[k], err_msg=k)
    assert d.hz == float(ref["hz"])
    assert list(d.glsizes) == list(ref["glsizes"]) == list(d.mysizes)


def test_domain_init_matches_oracle_and_roundtrips(lib, tmp_path):
    case = ic.plane_couette(10, 8, 8, 2000.0)
    d0 = ic.write_ic(case, str(tmp_path / "ic"))
    d = abi.DomainT()
    assert lib.domain_init(d0.encode(), C.byref(d)) == 0
    o = tn.load_domain(d0)
    nx = o.nx
    np.testing.assert_array_equal(np.ctypeslib.as_array(d.hxxf, shape=(nx + 1,)), o.hxxf[1:nx + 2])
    np.testing.assert_array_equal(np.ctypeslib.as_array(d.hxxc, shape=(nx + 2,)), o.hxxc)
    np.testing.assert_array_equal(np.ctypeslib.as_array(d.jdxc, shape=(nx + 2,)), o.jdxc)
    out = tmp_path / "save"
    out.mkdir()
    assert lib.domain_save(str(out).encode(), C.byref(d)) == 0
    for n in ("is_curved", "glsizes", "lengths", "xf", "xc"):
        a, b = np.load(out / f"{n}.npy"), np.load(os.path.join(d0, f"{n}.npy"))
        assert a.dtype == b.dtype and a.shape == b.shape
        np.testing.assert_array_equal(a, b)


def test_fluid_save_layout(lib, tmp_path):
    """fluid_save writes (nz, ny, nx+adds) NPYs without y/z halos (src/array.c:155-222)."""
    case = ic.taylor_couette(6, 8, 4, 3400.0)
    d0 = ic.write_ic(case, str(tmp_path / "ic"))
    d = abi.DomainT()
    assert lib.domain_init(d0.encode(), C.byref(d)) == 0
    fl = abi.FluidT()
    keep = []
    for n in ("ux", "uy", "uz", "p", "t"):
        a = np.load(os.path.join(d0, n + ".npy"))
        full = np.zeros((case.nz + 2, case.ny + 2, a.shape[2]))
        full[1:-1, 1:-1, :] = a
        keep.append(full)
        nadds = ((C.c_int * 2) * 3)((0, 1) if n == "ux" else (1, 1), (1, 1), (1, 1))
        arr = getattr(fl, n)
        arr.size = 8
        arr.nadds = C.cast(nadds, C.POINTER(C.c_int * 2))
        arr.datasize = full.nbytes
        arr.data = full.ctypes.data
        keep.append(nadds)
    fl.Re, fl.Pr = 3400.0, 1.0
    out = tmp_path / "save"
    out.mkdir()
    assert lib.fluid_save(str(out).encode(), C.byref(d), C.byref(fl)) == 0
    for n in ("ux", "uy", "uz", "p", "t"):
        np.testing.assert_array_equal(np.load(out / f"{n}.npy"), np.load(os.path.join(d0, n + ".npy")))
    assert float(np.load(out / "Re.npy")) == 3400.0


def test_startup_errors_are_reported(lib, tmp_path):
    d = abi.DomainT()
    assert lib.domain_init(b"/nonexistent/dir", C.byref(d)) != 0
    assert "No such file" in abi.last_error(lib)
    case = ic.taylor_couette(6, 8, 4, 3400.0)
    d0 = ic.write_ic(case, str(tmp_path / "ic"))
    np.save(os.path.join(d0, "xf.npy"), np.zeros(3, dtype=np.float32))        # wrong dtype and shape
    assert lib.domain_init(d0.encode(), C.byref(d)) != 0
    assert "dtype" in abi.last_error(lib)
    np.save(os.path.join(d0, "xf.npy"), np.zeros(3))                          # wrong shape
    assert lib.domain_init(d0.encode(), C.byref(d)) != 0
    assert "shape" in abi.last_error(lib)


def test_params_roundtrip(lib):
    p = abi.ParamsT(-0.5, 0.5, 1.0, 0.0, 1, 1, 1, 0.3, 0.9)
    assert lib.tcgpu_set_params(C.byref(p)) == 0
    q = abi.ParamsT()
    assert lib.tcgpu_get_params(C.byref(q)) == 0
    assert (q.uy_xm, q.uy_xp, q.t_xm, q.implicit_z, q.coef_dt_adv) == (-0.5, 0.5, 1.0, 1, 0.3)
    default = abi.ParamsT(1.0, 0.0, 0.5, -0.5, 1, 0, 0, -1.0, -1.0)
    lib.tcgpu_set_params(C.byref(default))


def test_domain_checks_single_rank_only(lib, tmp_path):
    case = ic.taylor_couette(6, 8, 4, 3400.0)
    d0 = ic.write_ic(case, str(tmp_path / "ic"))
    d = abi.DomainT()
    assert lib.domain_init(d0.encode(), C.byref(d)) == 0
    d.mysizes[1] = 4          # a decomposed domain is refused before any GPU work
    fl = abi.FluidT()
    dt = C.c_double()
    assert lib.decide_dt(C.byref(d), C.byref(fl), C.byref(dt)) != 0
    assert "single rank" in abi.last_error(lib)


def test_storage_selection_is_validated(lib):
    """tcgpu_set_storage takes 8 or 4 bytes per stored value and sets the
    storage of contexts created afterwards (no device needed)."""
    assert lib.tcgpu_get_storage(None) == 8
    assert lib.tcgpu_set_storage(3) != 0
    assert "8 or 4" in abi.last_error(lib)
    try:
        assert lib.tcgpu_set_storage(4) == 0
        assert lib.tcgpu_get_storage(None) == 4
    finally:
        assert lib.tcgpu_set_storage(8) == 0
    assert lib.tcgpu_get_storage(None) == 8
