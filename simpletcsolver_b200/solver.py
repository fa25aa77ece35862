"""Host-side driver of libtcgpu.so, mirroring the reference's start-up and time
loop (src/main.c:22-128): domain_init, fluid_init, then integrate() per step.

Everything numeric runs in the CUDA library; this module only owns the
domain_t / fluid_t structures, environment/parameter plumbing and numpy views
of the host arrays.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi
from .ic import Case, case_env

FIELD_BITS = {"ux": abi.UX, "uy": abi.UY, "uz": abi.UZ, "p": abi.P, "psi": abi.PSI, "t": abi.T}


def params_of(case: Case) -> abi.ParamsT:
    return abi.ParamsT(case.uy_xm, case.uy_xp, case.t_xm, case.t_xp,
                       int(case.implicit[0]), int(case.implicit[1]), int(case.implicit[2]),
                       case.coef_dt_adv, case.coef_dt_dif)


class SolverError(RuntimeError):
    pass


class Solver:
    """One domain + fluid held by the library; host arrays in the reference layout."""

    def __init__(self, lib, domain: abi.DomainT, fluid: abi.FluidT):
        self.lib = lib
        self.domain = domain
        self.fluid = fluid
        self.nx, self.ny, self.nz = (int(v) for v in domain.glsizes)

    # ---------------------------------------------------------------- set-up
    @classmethod
    def from_ic(cls, dirname: str, case: Case | None = None, Re: float | None = None, Pr: float | None = None,
                params: abi.ParamsT | None = None, lib=None, coherence: int = 0, storage: int = 8) -> "Solver":
        """storage: bytes per stored value of ux, uy, uz, t, the source terms and
        the spectra on the device (8, or 4 for the FP32-storage mode)."""
        lib = lib or abi.load()
        env = {}
        if case is not None:
            env.update(case_env(case))
            params = params or params_of(case)
        if Re is not None:
            env["Re"] = repr(float(Re))
        if Pr is not None:
            env["Pr"] = repr(float(Pr))
        os.environ.update(env)
        if params is not None:
            lib.tcgpu_set_params(C.byref(params))
        domain = abi.DomainT()
        fluid = abi.FluidT()
        if lib.domain_init(dirname.encode(), C.byref(domain)) != 0:
            raise SolverError(f"domain_init failed: {abi.last_error(lib)}")
        if lib.fluid_init(dirname.encode(), C.byref(domain), C.byref(fluid)) != 0:
            raise SolverError(f"fluid_init failed: {abi.last_error(lib)}")
        s = cls(lib, domain, fluid)
        previous = lib.tcgpu_get_storage(None)
        s._check(lib.tcgpu_set_storage(storage), "set_storage")
        try:
            s.set_coherence(coherence)   # creates the device context with that storage
        finally:
            lib.tcgpu_set_storage(previous)
        return s

    @classmethod
    def from_case(cls, case: Case, dirname: str, lib=None, coherence: int = 0, storage: int = 8) -> "Solver":
        """The case's seeded initial field generated on the device
        (tcgpu_fluid_init_generated); only the small domain files are written
        to dirname (ic.write_domain), no field NPYs."""
        from .ic import write_domain
        lib = lib or abi.load()
        os.environ.update(case_env(case))
        lib.tcgpu_set_params(C.byref(params_of(case)))
        write_domain(case, dirname)
        domain = abi.DomainT()
        fluid = abi.FluidT()
        if lib.domain_init(dirname.encode(), C.byref(domain)) != 0:
            raise SolverError(f"domain_init failed: {abi.last_error(lib)}")
        s = cls(lib, domain, fluid)
        previous = lib.tcgpu_get_storage(None)
        s._check(lib.tcgpu_set_storage(storage), "set_storage")
        try:
            icp = abi.IcT(case.seed, case.noise_u, case.noise_t)
            s._check(lib.tcgpu_fluid_init_generated(C.byref(domain), C.byref(fluid), C.byref(icp)),
                     "fluid_init_generated")
        finally:
            lib.tcgpu_set_storage(previous)
        s.set_coherence(coherence)
        return s

    @property
    def storage(self) -> int:
        return self.lib.tcgpu_get_storage(C.byref(self.fluid))

    def _check(self, rc: int, what: str):
        if rc != 0:
            raise SolverError(f"{what} failed: {abi.last_error(self.lib)}")

    def set_coherence(self, flags: int):
        self._check(self.lib.tcgpu_set_coherence(C.byref(self.domain), C.byref(self.fluid), flags), "set_coherence")

    # ---------------------------------------------------------------- views
    def array(self, arr: abi.ArrayT, rowlen: int, nj: int, nk: int) -> np.ndarray:
        n = rowlen * nj * nk
        buf = (C.c_double * n).from_address(arr.data)
        return np.frombuffer(buf, dtype=np.float64).reshape(nk, nj, rowlen)

    def field(self, name: str) -> np.ndarray:
        """Host array of a field, shape (nz+2, ny+2, rowlen), [k, j, i]."""
        rowlen = self.nx + 1 if name == "ux" else self.nx + 2
        return self.array(getattr(self.fluid, name), rowlen, self.ny + 2, self.nz + 2)

    def src(self, var: str, slot: int) -> np.ndarray:
        rowlen = self.nx - 1 if var == "ux" else self.nx
        arrs = getattr(self.fluid, "src" + var if var != "t" else "srct")
        return self.array(arrs[slot], rowlen, self.ny, self.nz)

    def tensor(self, name: str) -> np.ndarray:
        face = name in ("lxy", "lxz", "lyx0", "lyx1", "lzx")
        return self.array(getattr(self.fluid, name), self.nx + 1 if face else self.nx, self.ny + 2, self.nz + 2)

    # ---------------------------------------------------------------- reference entry points
    def decide_dt(self) -> float:
        dt = C.c_double(0.)
        self._check(self.lib.decide_dt(C.byref(self.domain), C.byref(self.fluid), C.byref(dt)), "decide_dt")
        return dt.value

    def integrate(self) -> float:
        dt = C.c_double(0.)
        self._check(self.lib.integrate(C.byref(self.domain), C.byref(self.fluid), C.byref(dt)), "integrate")
        return dt.value

    def predict(self, rk: int, dt: float):
        self._check(self.lib.fluid_predict_field(C.byref(self.domain), rk, dt, C.byref(self.fluid)), "predict")

    def compute_potential(self, rk: int, dt: float):
        self._check(self.lib.fluid_compute_potential(C.byref(self.domain), rk, dt, C.byref(self.fluid)),
                    "compute_potential")

    def correct_velocity(self, rk: int, dt: float):
        self._check(self.lib.fluid_correct_velocity(C.byref(self.domain), rk, dt, C.byref(self.fluid)),
                    "correct_velocity")

    def update_pressure(self, rk: int, dt: float):
        self._check(self.lib.fluid_update_pressure(C.byref(self.domain), rk, dt, C.byref(self.fluid)),
                    "update_pressure")

    # ---------------------------------------------------------------- residency
    def push(self, mask: int = abi.FIELDS):
        self._check(self.lib.tcgpu_push(C.byref(self.domain), C.byref(self.fluid), mask), "push")

    def pull(self, mask: int = abi.FIELDS):
        self._check(self.lib.tcgpu_pull(C.byref(self.domain), C.byref(self.fluid), mask), "pull")

    def run(self, nsteps: int) -> np.ndarray:
        dts = np.zeros(nsteps)
        self._check(self.lib.tcgpu_run(C.byref(self.domain), C.byref(self.fluid), nsteps,
                                       dts.ctypes.data_as(abi.c_double_p)), "run")
        return dts

    def diagnostics(self) -> dict:
        out = (C.c_double * 9)()
        self._check(self.lib.tcgpu_diagnostics(C.byref(self.domain), C.byref(self.fluid), out), "diagnostics")
        keys = ("divmax", "injection_u", "injection_t", "dissipation_u", "dissipation_t",
                "energy_ux", "energy_uy", "energy_uz", "energy_t")
        return dict(zip(keys, list(out)))

    def log_quantities(self) -> dict:
        """The nine logging quantities with the reference's semantics (tensors
        of the last predict's input fields; src/logging/*.c after integrate())."""
        out = (C.c_double * 9)()
        self._check(self.lib.tcgpu_log_quantities(C.byref(self.domain), C.byref(self.fluid), out), "log_quantities")
        keys = ("divmax", "injection_u", "injection_t", "dissipation_u", "dissipation_t",
                "energy_ux", "energy_uy", "energy_uz", "energy_t")
        return dict(zip(keys, list(out)))

    def radial_slab(self, name: str, i0: int, count: int) -> np.ndarray:
        """Device values of a field at radial indices i0 .. i0+count-1 over the
        interior j, k: array [k, j, c]."""
        out = np.zeros((self.nz, self.ny, count))
        self._check(self.lib.tcgpu_radial_slab(C.byref(self.domain), C.byref(self.fluid), FIELD_BITS[name], i0, count,
                                               out.ctypes.data_as(abi.c_double_p)), "radial_slab")
        return out

    # ---------------------------------------------------------------- statistics (src/statistics.c)
    STAT_NAMES = ("ux1", "ux2", "uy1", "uy2", "uz1", "uz2", "adv", "dif")

    def stats_collect(self):
        self._check(self.lib.tcgpu_statistics_collect(C.byref(self.domain), C.byref(self.fluid)), "statistics_collect")

    def stats_reset(self):
        self._check(self.lib.tcgpu_statistics_reset(C.byref(self.domain), C.byref(self.fluid)), "statistics_reset")

    def stats(self) -> tuple[int, dict]:
        """(samples, {name: array [k, j, i]}) of the device accumulators."""
        arrays = {}
        ptrs = (abi.c_double_p * 8)()
        for s, name in enumerate(self.STAT_NAMES):
            row = self.nx + 2 if name[:2] in ("uy", "uz") else self.nx + 1
            arrays[name] = np.zeros((self.nz, self.ny, row))
            ptrs[s] = arrays[name].ctypes.data_as(abi.c_double_p)
        num = C.c_size_t(0)
        self._check(self.lib.tcgpu_statistics_get(C.byref(self.domain), C.byref(self.fluid), C.byref(num), ptrs),
                    "statistics_get")
        return int(num.value), arrays

    def stats_save(self, dirname: str):
        os.makedirs(dirname, exist_ok=True)
        self._check(self.lib.tcgpu_statistics_save(dirname.encode(), C.byref(self.domain), C.byref(self.fluid)),
                    "statistics_save")

    def mean_uy(self) -> np.ndarray:
        """Mean azimuthal velocity profile uy(r), i = 0..nx+1, over j, k and the samples."""
        out = np.zeros(self.nx + 2)
        self._check(self.lib.tcgpu_statistics_mean_uy(C.byref(self.domain), C.byref(self.fluid),
                                                      out.ctypes.data_as(abi.c_double_p)), "statistics_mean_uy")
        return out

    def save(self, dirname: str, step: int = 0, time: float = 0.0):
        """Reference save layout (src/save.c:74-110): step, time, domain, fluid."""
        os.makedirs(dirname, exist_ok=True)
        np.save(os.path.join(dirname, "step.npy"), np.array(step, dtype=np.uint64))
        np.save(os.path.join(dirname, "time.npy"), np.array(time, dtype=np.float64))
        self._check(self.lib.domain_save(dirname.encode(), C.byref(self.domain)), "domain_save")
        self._check(self.lib.fluid_save(dirname.encode(), C.byref(self.domain), C.byref(self.fluid)), "fluid_save")

    def release(self):
        self.lib.tcgpu_release(C.byref(self.fluid))
