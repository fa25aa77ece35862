"""Generate the golden fixtures under tests/golden/ from the reference itself.

The reference's own C sources, compiled against the single-rank shims by
oracle/Makefile (oracle/_ref/libtcref_<cfg>.so), are driven through ctypes:

  <cfg>.npz   initial fields of a small seeded case, the reference's fields
              after N calls of integrate() (src/integrate.c:9-35), the last dt
              and time, and the reference's logging quantities of the final
              fields (src/logging/*.c, with the velocity-gradient tensors
              recomputed from those fields by the reference's compute_l*)
  tdm.npz     random diagonally dominant systems (real/complex, periodic or
              not) and the reference tdm.solve() answers (src/tdm.c)

Each configuration runs in its own process because the reference keeps its
solver state in function-local statics bound to the first grid it sees.

    python tests/golden/make_golden.py            # all fixtures
"""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from simpletcsolver_b200 import abi, ic  # noqa: E402

CASES = {
    # name: (build, case, steps)
    "tc": ("tc", ic.taylor_couette(12, 16, 8, 3400.0), 20),
    "tcexp": ("tcexp", ic.taylor_couette(8, 16, 8, 3400.0, implicit=(False, False, False)), 10),
    "planar": ("planar", ic.plane_couette(8, 8, 8, 2000.0), 10),
}
FIELDS = ("ux", "uy", "uz", "p", "t")


def ref_lib(build: str):
    path = os.path.join(ROOT, "oracle", "_ref", f"libtcref_{build}.so")
    lib = C.CDLL(path)
    abi.bind_reference_api(lib)
    return lib


def host_view(arr: abi.ArrayT, shape):
    n = int(np.prod(shape))
    return np.frombuffer((C.c_double * n).from_address(arr.data), dtype=np.float64).reshape(shape).copy()


def run_one(name: str, out: str):
    build, case, steps = CASES[name]
    os.environ.update(ic.case_env(case))
    lib = ref_lib(build)
    with tempfile.TemporaryDirectory() as d0:
        ic.write_ic(case, d0)
        ics = {n: np.load(os.path.join(d0, n + ".npy")) for n in
               ("ux", "uy", "uz", "p", "t", "xf", "xc", "glsizes", "lengths", "is_curved")}
        domain = abi.DomainT()
        fluid = abi.FluidT()
        assert lib.domain_init(d0.encode(), C.byref(domain)) == 0
        assert lib.fluid_init(d0.encode(), C.byref(domain), C.byref(fluid)) == 0
        dt = C.c_double(0.)
        time = 0.0
        for _ in range(steps):
            assert lib.integrate(C.byref(domain), C.byref(fluid), C.byref(dt)) == 0
            time += dt.value
        nx, ny, nz = case.nx, case.ny, case.nz
        final = {}
        for n in FIELDS:
            row = nx + 1 if n == "ux" else nx + 2
            full = host_view(getattr(fluid, n), (nz + 2, ny + 2, row))
            final["ref_" + n] = full
        # logging quantities of the final fields
        for f in ("compute_lxx", "compute_lxy", "compute_lxz", "compute_lyx", "compute_lyy",
                  "compute_lyz", "compute_lzx", "compute_lzy", "compute_lzz"):
            getattr(lib, f)(C.byref(domain), C.byref(fluid))
        logs = {}
        with tempfile.TemporaryDirectory() as lg:
            for key in ("divergence", "injection", "dissipation", "total_energy"):
                fn = os.path.join(lg, key + ".dat")
                getattr(lib, "logging_check_" + key)(fn.encode(), C.byref(domain), C.c_double(time), C.byref(fluid))
                logs[key] = [float(v) for v in open(fn).read().split()[1:]]
    meta = dict(case=case.__dict__ | {"implicit": list(case.implicit)}, steps=steps, dt_last=dt.value, time=time,
                logs=logs, build=build)
    np.savez_compressed(out, meta=json.dumps(meta), **{"ic_" + k: v for k, v in ics.items()}, **final)


def make_tdm(out: str):
    lib = ref_lib("tc")
    tdm = abi.tdm_vtable(lib)
    rng = np.random.default_rng(1234)
    arrays = {}
    for periodic in (False, True):
        for cplx in (False, True):
            n, nrhs = 13, 5
            info = abi.TdmInfoP()
            assert tdm.construct(n, nrhs, periodic, cplx, C.byref(info)) == 0
            ptr = abi.c_double_p()
            coefs = {}
            for nm, getter in (("l", tdm.get_l), ("c", tdm.get_c), ("u", tdm.get_u)):
                getter(info, C.byref(ptr))
                v = rng.uniform(-1.0, 1.0, n) if nm != "c" else rng.uniform(2.5, 4.0, n) * rng.choice([-1.0, 1.0], n)
                np.ctypeslib.as_array(ptr, shape=(n,))[:] = v
                coefs[nm] = v.copy()
            q = rng.standard_normal((nrhs, n, 2) if cplx else (nrhs, n))
            data = np.ascontiguousarray(q.copy())
            assert tdm.solve(info, data.ctypes.data_as(C.c_void_p)) == 0
            tdm.destruct(info)
            key = f"{'p' if periodic else 'n'}{'c' if cplx else 'r'}"
            for nm, v in coefs.items():
                arrays[f"{key}_{nm}"] = v
            arrays[f"{key}_q"] = q
            arrays[f"{key}_x"] = data
    np.savez_compressed(out, **arrays)


def main():
    if len(sys.argv) > 2 and sys.argv[1] == "--one":
        name = sys.argv[2]
        if name == "tdm":
            make_tdm(os.path.join(HERE, "tdm.npz"))
        else:
            run_one(name, os.path.join(HERE, f"{name}.npz"))
        return
    for name in list(CASES) + ["tdm"]:
        subprocess.run([sys.executable, __file__, "--one", name], check=True, cwd=ROOT,
                       stdout=subprocess.DEVNULL)
        print("wrote", name)


if __name__ == "__main__":
    main()
