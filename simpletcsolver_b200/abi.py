"""ctypes view of the C ABI in include/tcgpu.h.

The structures are layout-compatible with the reference's domain_t, array_t
and fluid_t (include/domain.h, include/array.h, include/fluid.h), so the same
Python objects drive libtcgpu.so and the reference's own library.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "libtcgpu.so")
HEADER = os.path.join(ROOT, "include", "tcgpu.h")

c_double_p = C.POINTER(C.c_double)


class ArrayT(C.Structure):
    _fields_ = [("size", C.c_size_t), ("nadds", C.POINTER(C.c_int * 2)),
                ("datasize", C.c_size_t), ("data", C.c_void_p)]


class DomainT(C.Structure):
    _fields_ = [("info", C.c_void_p), ("is_curved", C.c_bool),
                ("glsizes", C.c_size_t * 3), ("mysizes", C.c_size_t * 3), ("offsets", C.c_size_t * 3),
                ("lengths", C.c_double * 3),
                ("xf", c_double_p), ("xc", c_double_p), ("jdxf", c_double_p), ("jdxc", c_double_p),
                ("hxxf", c_double_p), ("hxxc", c_double_p), ("hyxf", c_double_p), ("hyxc", c_double_p),
                ("hz", C.c_double)]


class FluidT(C.Structure):
    _fields_ = [("ux", ArrayT), ("uy", ArrayT), ("uz", ArrayT), ("p", ArrayT), ("psi", ArrayT), ("t", ArrayT),
                ("srcux", ArrayT * 3), ("srcuy", ArrayT * 3), ("srcuz", ArrayT * 3), ("srct", ArrayT * 3),
                ("lxx", ArrayT), ("lyx0", ArrayT), ("lyx1", ArrayT), ("lxy", ArrayT), ("lzx", ArrayT),
                ("lxz", ArrayT), ("lyy0", ArrayT), ("lyy1", ArrayT), ("lzy", ArrayT), ("lyz", ArrayT),
                ("lzz", ArrayT), ("Re", C.c_double), ("Pr", C.c_double)]


class IcT(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("noise_u", C.c_double), ("noise_t", C.c_double)]


class ParamsT(C.Structure):
    _fields_ = [("uy_xm", C.c_double), ("uy_xp", C.c_double), ("t_xm", C.c_double), ("t_xp", C.c_double),
                ("implicit_x", C.c_int), ("implicit_y", C.c_int), ("implicit_z", C.c_int),
                ("coef_dt_adv", C.c_double), ("coef_dt_dif", C.c_double)]


TdmInfoP = C.c_void_p


class TdmT(C.Structure):
    _fields_ = [("construct", C.CFUNCTYPE(C.c_int, C.c_int, C.c_int, C.c_bool, C.c_bool, C.POINTER(TdmInfoP))),
                ("get_l", C.CFUNCTYPE(C.c_int, TdmInfoP, C.POINTER(c_double_p))),
                ("get_c", C.CFUNCTYPE(C.c_int, TdmInfoP, C.POINTER(c_double_p))),
                ("get_u", C.CFUNCTYPE(C.c_int, TdmInfoP, C.POINTER(c_double_p))),
                ("get_size", C.CFUNCTYPE(C.c_int, TdmInfoP, C.POINTER(C.c_int))),
                ("get_nrhs", C.CFUNCTYPE(C.c_int, TdmInfoP, C.POINTER(C.c_int))),
                ("solve", C.CFUNCTYPE(C.c_int, TdmInfoP, C.c_void_p)),
                ("destruct", C.CFUNCTYPE(C.c_int, TdmInfoP))]


# field / coherence bits of include/tcgpu.h
UX, UY, UZ, P, PSI, T = 1, 2, 4, 8, 16, 32
FIELDS = 63
SRCS, TENSORS = 64, 128
SYNC_SRCS, SYNC_TENSORS, NO_COHERENCE, PIN_HOST = 1, 2, 4, 8

_SIGS = {
    "integrate": (C.c_int, [C.POINTER(DomainT), C.POINTER(FluidT), c_double_p]),
    "decide_dt": (C.c_int, [C.POINTER(DomainT), C.POINTER(FluidT), c_double_p]),
    "fluid_predict_field": (C.c_int, [C.POINTER(DomainT), C.c_size_t, C.c_double, C.POINTER(FluidT)]),
    "fluid_compute_potential": (C.c_int, [C.POINTER(DomainT), C.c_size_t, C.c_double, C.POINTER(FluidT)]),
    "fluid_correct_velocity": (C.c_int, [C.POINTER(DomainT), C.c_size_t, C.c_double, C.POINTER(FluidT)]),
    "fluid_update_pressure": (C.c_int, [C.POINTER(DomainT), C.c_size_t, C.c_double, C.POINTER(FluidT)]),
    "fluid_compute_momentum_diffusivity": (C.c_double, [C.POINTER(FluidT)]),
    "fluid_compute_scalar_diffusivity": (C.c_double, [C.POINTER(FluidT)]),
    "fluid_init": (C.c_int, [C.c_char_p, C.POINTER(DomainT), C.POINTER(FluidT)]),
    "fluid_save": (C.c_int, [C.c_char_p, C.POINTER(DomainT), C.POINTER(FluidT)]),
    "domain_init": (C.c_int, [C.c_char_p, C.POINTER(DomainT)]),
    "domain_save": (C.c_int, [C.c_char_p, C.POINTER(DomainT)]),
}
for _n in ("ux", "uy", "uz", "p", "psi", "t"):
    _SIGS[f"fluid_update_boundaries_{_n}"] = (C.c_int, [C.POINTER(DomainT), C.POINTER(ArrayT)])

_EXT_SIGS = {
    "tcgpu_set_params": (C.c_int, [C.POINTER(ParamsT)]),
    "tcgpu_get_params": (C.c_int, [C.POINTER(ParamsT)]),
    "tcgpu_set_coherence": (C.c_int, [C.POINTER(DomainT), C.POINTER(FluidT), C.c_uint]),
    "tcgpu_push": (C.c_int, [C.POINTER(DomainT), C.POINTER(FluidT), C.c_uint]),
    "tcgpu_pull": (C.c_int, [C.POINTER(DomainT), C.POINTER(FluidT), C.c_uint]),
    "tcgpu_run": (C.c_int, [C.POINTER(DomainT), C.POINTER(FluidT), C.c_int, c_double_p]),
    "tcgpu_diagnostics": (C.c_int, [C.POINTER(DomainT), C.POINTER(FluidT), C.c_double * 9]),
    "tcgpu_log_quantities": (C.c_int, [C.POINTER(DomainT), C.POINTER(FluidT), C.c_double * 9]),
    "tcgpu_fluid_init_generated": (C.c_int, [C.POINTER(DomainT), C.POINTER(FluidT), C.POINTER(IcT)]),
    "tcgpu_radial_slab": (C.c_int, [C.POINTER(DomainT), C.POINTER(FluidT), C.c_uint, C.c_int, C.c_int,
                                    c_double_p]),
    "tcgpu_statistics_collect": (C.c_int, [C.POINTER(DomainT), C.POINTER(FluidT)]),
    "tcgpu_statistics_reset": (C.c_int, [C.POINTER(DomainT), C.POINTER(FluidT)]),
    "tcgpu_statistics_get": (C.c_int, [C.POINTER(DomainT), C.POINTER(FluidT), C.POINTER(C.c_size_t),
                                       c_double_p * 8]),
    "tcgpu_statistics_save": (C.c_int, [C.c_char_p, C.POINTER(DomainT), C.POINTER(FluidT)]),
    "tcgpu_statistics_mean_uy": (C.c_int, [C.POINTER(DomainT), C.POINTER(FluidT), c_double_p]),
    "tcgpu_release": (C.c_int, [C.POINTER(FluidT)]),
    "tcgpu_set_storage": (C.c_int, [C.c_int]),
    "tcgpu_get_storage": (C.c_int, [C.POINTER(FluidT)]),
    "tcgpu_last_error": (C.c_char_p, []),
    "tcgpu_selftest_wait": (C.c_int, [c_double_p]),
    "tcgpu_set_device": (C.c_int, [C.c_int]),
    "tcgpu_run_timed": (C.c_int, [C.POINTER(DomainT), C.POINTER(FluidT), C.c_int, C.c_int, c_double_p,
                                  C.POINTER(C.c_float), C.c_double * 12, C.c_int * 12]),
    "tcgpu_tdm_solve_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_bool, C.c_bool, c_double_p, c_double_p, c_double_p,
                                          C.c_void_p]),
    "tcgpu_stream": (C.c_void_p, [C.POINTER(DomainT), C.POINTER(FluidT)]),
    "tcgpu_coarsen": (C.c_int, [C.POINTER(DomainT), C.POINTER(FluidT), C.POINTER(DomainT), C.POINTER(FluidT)]),
    "tcgpu_closure_input": (C.c_int, [C.POINTER(DomainT), C.POINTER(FluidT), C.c_double * 3, C.c_int, C.c_void_p]),
    "tcgpu_closure_target": (C.c_int, [C.POINTER(DomainT), C.POINTER(FluidT), C.POINTER(FluidT), C.c_double,
                                       C.c_void_p]),
    "tcgpu_set_forcing": (C.c_int, [C.POINTER(DomainT), C.POINTER(FluidT), C.c_void_p, C.c_int, C.c_double * 3]),
    "tcgpu_nn_pack_weights": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                        C.c_void_p]),
    "tcgpu_nn_conv3": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "tcgpu_nn_wgrad_workspace": (C.c_size_t, [C.c_int, C.c_int, C.c_int, C.c_int]),
    "tcgpu_nn_conv3_wgrad": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_void_p, C.c_size_t,
                                       C.c_void_p]),
    "tcgpu_nn_mse": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_int, C.c_int, C.c_void_p,
                               C.c_void_p, C.c_void_p]),
    "tcgpu_nn_adam": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_float, C.c_float,
                                C.c_float, C.c_float, C.c_int, C.c_void_p]),
    "tcgpu_nn_status": (C.c_int, [C.c_int]),
    "tcgpu_nn_last_error": (C.c_char_p, []),
}


def declared_symbols(header: str = HEADER):
    """Function and object names declared in include/*.h."""
    src = open(header).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = set(re.findall(r"^\s*(?:extern\s+)?(?:const\s+)?[\w\s\*]+?\b(\w+)\s*\(", src, flags=re.M))
    names |= set(re.findall(r"^\s*extern\s+const\s+\w+\s+(\w+)", src, flags=re.M))
    return sorted(n for n in names if n not in ("if", "defined", "int", "double", "void"))


def declared_functions(header: str = HEADER):
    """Top-level function declarations of include/*.h: name -> number of
    parameters (the function-pointer members of tdm_t are not top level)."""
    src = re.sub(r"/\*.*?\*/", "", open(header).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"^[ \t]*(?:extern\s+)?[A-Za-z_][\w \t\*]*?\b([A-Za-z_]\w*)\s*\(([^()]*)\)\s*;", src,
                         flags=re.M):
        params = " ".join(m.group(2).split())
        out[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def _bind(lib, sigs):
    for name, (res, args) in sigs.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args


def bind_reference_api(lib):
    """Attach argtypes for the reference's entry points (works for libtcref too)."""
    _bind(lib, _SIGS)
    return lib


_lib = None


def load(path: str | None = None):
    """Load libtcgpu.so. Raises if it has not been built: the solver has no
    CPU fallback."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"{p} is missing; build it with `python -m simpletcsolver_b200.build`")
    lib = C.CDLL(p)
    _bind(lib, _SIGS)
    _bind(lib, _EXT_SIGS)
    if path is None:
        _lib = lib
    return lib


def tdm_vtable(lib) -> TdmT:
    return TdmT.in_dll(lib, "tdm")


def last_error(lib) -> str:
    return lib.tcgpu_last_error().decode()
