"""CPU restatement of SimpleTCSolver's RK3 time step in numpy (FP64).

TEST INFRASTRUCTURE ONLY. This module is the oracle that the CUDA library is
checked against; it is imported by tests/, by the package's smoke check and by
bench.py's CPU-baseline leg, never by the product path. It is itself pinned
against the reference compiled from its own sources (oracle/Makefile) in
tests/test_oracle.py.

Layout: every field is a numpy array A[k, j, i] holding the reference's index
space including halos, i.e. i, j, k run over 0..n+1 and A[k, j, i] is the
reference's A(i, j, k) (array_macros/fluid/*.h). ux keeps an unused i=0 column
so that its reference indices (1..nx+1) map directly. RK source terms use the
reference's own packed interior layout (srcux: i=2..nx, others i=1..nx).
Metric arrays are indexed by the reference i as well (unused entries zero).

Expressions keep the reference's operand order so that, FFTs aside, results
agree to the last bits or nearly so.
"""
from __future__ import annotations

import dataclasses
import os

import numpy as np

# Wray RK3, src/runge_kutta.c:8-15
RK_A = (32.0 / 60.0, 25.0 / 60.0, 45.0 / 60.0)
RK_B = (0.0 / 60.0, -17.0 / 60.0, -25.0 / 60.0)
RK_G = tuple(a + b for a, b in zip(RK_A, RK_B))

DBL_EPSILON = np.finfo(np.float64).eps


@dataclasses.dataclass
class Params:
    """Compile-time constants of the reference (src/param/*.c), runtime here."""
    uy_xm: float = 1.0
    uy_xp: float = 0.0
    t_xm: float = 0.5
    t_xp: float = -0.5
    implicit: tuple = (True, False, False)
    coef_dt_adv: float = 0.4
    coef_dt_dif: float = 1.0


@dataclasses.dataclass
class Domain:
    """domain_t (include/domain.h:23-37) with metric arrays, src/domain.c:259-357."""
    is_curved: bool
    nx: int
    ny: int
    nz: int
    lengths: np.ndarray
    xf: np.ndarray    # reference i = 1..nx+1 at index i
    xc: np.ndarray    # i = 0..nx+1
    hxxf: np.ndarray
    hxxc: np.ndarray
    hyxf: np.ndarray
    hyxc: np.ndarray
    jdxf: np.ndarray
    jdxc: np.ndarray
    hz: float


def make_domain(is_curved, glsizes, lengths, xf_npy, xc_npy) -> Domain:
    nx, ny, nz = (int(v) for v in glsizes)
    lengths = np.asarray(lengths, dtype=np.float64)
    xf = np.zeros(nx + 2)
    xf[1:] = xf_npy                      # XF(I) = xf[I-1] in the reference
    xc = np.asarray(xc_npy, dtype=np.float64).copy()
    hxxf = np.zeros(nx + 2)
    hxxc = np.zeros(nx + 2)
    hyxf = np.zeros(nx + 2)
    hyxc = np.zeros(nx + 2)
    jdxf = np.zeros(nx + 2)
    jdxc = np.zeros(nx + 2)
    for i in range(1, nx + 2):           # domain.c:265-268
        hxxf[i] = xc[i] - xc[i - 1]
    hxxc[0] = 0.5 * xf[2] - 0.5 * xf[1]  # domain.c:280-284
    for i in range(1, nx + 1):
        hxxc[i] = xf[i + 1] - xf[i]
    hxxc[nx + 1] = 0.5 * xf[nx + 1] - 0.5 * xf[nx]
    ly = lengths[1]
    for i in range(1, nx + 2):           # domain.c:297-300
        hyxf[i] = xf[i] * ly / ny if is_curved else ly / ny
    for i in range(0, nx + 2):           # domain.c:314-317
        hyxc[i] = xc[i] * ly / ny if is_curved else ly / ny
    hz = lengths[2] / nz
    for i in range(1, nx + 2):           # domain.c:330-333
        jdxf[i] = hxxf[i] * hyxf[i] * hz
    for i in range(0, nx + 2):           # domain.c:346-349
        jdxc[i] = hxxc[i] * hyxc[i] * hz
    return Domain(bool(is_curved), nx, ny, nz, lengths, xf, xc, hxxf, hxxc, hyxf, hyxc, jdxf, jdxc, hz)


def load_domain(dirname) -> Domain:
    """domain_load + domain_init (src/domain.c:28-55, 389-432)."""
    ld = lambda n: np.load(os.path.join(dirname, n + ".npy"))
    return make_domain(bool(ld("is_curved")), ld("glsizes"), ld("lengths"), ld("xf"), ld("xc"))


@dataclasses.dataclass
class Fluid:
    """fluid_t (include/fluid.h:18-36); src[v] = [alpha, beta] packed arrays."""
    ux: np.ndarray
    uy: np.ndarray
    uz: np.ndarray
    p: np.ndarray
    psi: np.ndarray
    t: np.ndarray
    src: dict
    Re: float
    Pr: float
    tensors: dict = dataclasses.field(default_factory=dict)


def full(d: Domain):
    return np.zeros((d.nz + 2, d.ny + 2, d.nx + 2))


def from_npy(d: Domain, name: str, arr: np.ndarray) -> np.ndarray:
    """NPY (nz, ny, nx+adds) -> halo array; src/array.c:124-152."""
    a = full(d)
    if name == "ux":
        a[1:-1, 1:-1, 1:] = arr
    else:
        a[1:-1, 1:-1, :] = arr
    return a


def to_npy(d: Domain, name: str, a: np.ndarray) -> np.ndarray:
    if name == "ux":
        return np.ascontiguousarray(a[1:-1, 1:-1, 1:])
    return np.ascontiguousarray(a[1:-1, 1:-1, :])


def make_fluid(d: Domain, fields: dict, Re: float, Pr: float, prm: Params) -> Fluid:
    """fluid_init (src/fluid/init.c:98-122): load, impose BCs and halos."""
    fl = Fluid(ux=from_npy(d, "ux", fields["ux"]), uy=from_npy(d, "uy", fields["uy"]),
               uz=from_npy(d, "uz", fields["uz"]), p=from_npy(d, "p", fields["p"]),
               psi=full(d), t=from_npy(d, "t", fields["t"]), Re=float(Re), Pr=float(Pr),
               src={v: [np.zeros(src_shape(d, v)), np.zeros(src_shape(d, v))] for v in ("ux", "uy", "uz", "t")})
    bc_ux(d, fl.ux)
    bc_uy(d, fl.uy, prm)
    bc_uz(d, fl.uz)
    bc_p(d, fl.p)
    bc_t(d, fl.t, prm)
    return fl


def load_fluid(d: Domain, dirname, Re, Pr, prm: Params) -> Fluid:
    fields = {n: np.load(os.path.join(dirname, n + ".npy")) for n in ("ux", "uy", "uz", "p", "t")}
    return make_fluid(d, fields, Re, Pr, prm)


def src_shape(d: Domain, v: str):
    return (d.nz, d.ny, d.nx - 1) if v == "ux" else (d.nz, d.ny, d.nx)


# ---------------------------------------------------------------- helpers

def V(d: Domain, a, ilo, ihi, di=0, dj=0, dk=0):
    """a(i+di, j+dj, k+dk) for i in [ilo, ihi], j in [1, ny], k in [1, nz]."""
    return a[1 + dk:d.nz + 1 + dk, 1 + dj:d.ny + 1 + dj, ilo + di:ihi + 1 + di]


def M(m, ilo, ihi, di=0):
    """metric m(i+di) for i in [ilo, ihi], broadcast along the last axis."""
    return m[ilo + di:ihi + 1 + di]


def halo_yz(a):
    """halo_communicate_in_y then _in_z with one rank (src/halo.c:18-142):
    periodic images, y first over all x and interior k, then whole z planes."""
    a[1:-1, 0, :] = a[1:-1, -2, :]
    a[1:-1, -1, :] = a[1:-1, 1, :]
    a[0, :, :] = a[-2, :, :]
    a[-1, :, :] = a[1, :, :]


def bc_ux(d, ux):      # src/fluid/boundary/ux.c:13-45
    ux[1:-1, 1:-1, 1] = 0.0
    ux[1:-1, 1:-1, d.nx + 1] = 0.0
    halo_yz(ux)


def bc_uy(d, uy, prm):  # src/fluid/boundary/uy.c:14-46
    uy[1:-1, 1:-1, 0] = prm.uy_xm
    uy[1:-1, 1:-1, d.nx + 1] = prm.uy_xp
    halo_yz(uy)


def bc_uz(d, uz):      # src/fluid/boundary/uz.c
    uz[1:-1, 1:-1, 0] = 0.0
    uz[1:-1, 1:-1, d.nx + 1] = 0.0
    halo_yz(uz)


def bc_p(d, p):        # src/fluid/boundary/p.c:13-45 (Neumann), also psi.c
    p[1:-1, 1:-1, 0] = p[1:-1, 1:-1, 1]
    p[1:-1, 1:-1, d.nx + 1] = p[1:-1, 1:-1, d.nx]
    halo_yz(p)


bc_psi = bc_p


def bc_t(d, t, prm):   # src/fluid/boundary/t.c
    t[1:-1, 1:-1, 0] = prm.t_xm
    t[1:-1, 1:-1, d.nx + 1] = prm.t_xp
    halo_yz(t)


def _rdiv(q, c):
    """q / c for a real divisor, componentwise when q is complex (C99 Annex G
    semantics of double _Complex / double, as the reference computes it)."""
    if np.iscomplexobj(q):
        return (q.real / c) + 1j * (q.imag / c)
    return q / c


def gtsv(l, c, u, q, singular_guard=True):
    """Thomas algorithm along axis 0 of q (src/tdm.c:17-50); l, c, u have
    length n along axis 0 and broadcast against q[i]. q is overwritten."""
    n = q.shape[0]
    v = np.empty((n,) + np.broadcast(c[0], q[0]).shape if np.ndim(c) > 1 else (n,))
    v[0] = u[0] / c[0]
    q[0] = _rdiv(q[0], c[0])
    for i in range(1, n - 1):
        val = 1.0 / (c[i] - l[i] * v[i - 1])
        v[i] = val * (u[i])
        q[i] = val * (q[i] - l[i] * q[i - 1])
    if n > 1:
        val = c[n - 1] - l[n - 1] * v[n - 2]
        good = np.abs(val) > DBL_EPSILON
        if np.ndim(good) == 0:
            q[n - 1] = (1.0 / val * (q[n - 1] - l[n - 1] * q[n - 2])) if good else 0.0
        else:
            with np.errstate(divide="ignore", invalid="ignore"):
                res = 1.0 / val * (q[n - 1] - l[n - 1] * q[n - 2])
            q[n - 1] = np.where(good, res, 0.0) if singular_guard else res
    for i in range(n - 2, -1, -1):
        q[i] -= v[i] * q[i + 1]
    return q


def tdm_periodic(l, c, u, q):
    """Periodic system via Sherman-Morrison on the reduced system
    (src/tdm.c:66-99); q along axis 0, coefficients broadcast."""
    n = q.shape[0]
    shp = np.broadcast(c[0], q[0]).shape
    q1 = np.zeros((n - 1,) + shp)
    q1[0] = -l[0]
    if n - 2 > 0:
        q1[n - 2] = -u[n - 2]
    gtsv(l[:n - 1], c[:n - 1], u[:n - 1], q1)
    q0 = q
    gtsv(l[:n - 1], c[:n - 1], u[:n - 1], q0[:n - 1])
    num = q0[n - 1] - u[n - 1] * q0[0] - l[n - 1] * q0[n - 2]
    den = c[n - 1] + u[n - 1] * q1[0] + l[n - 1] * q1[n - 2]
    with np.errstate(divide="ignore", invalid="ignore"):
        last = np.where(np.abs(den) < DBL_EPSILON, 0.0, _rdiv(num, den))
    q0[n - 1] = last
    q0[:n - 1] = q0[:n - 1] + q0[n - 1] * q1
    return q0


# ---------------------------------------------------------------- decide_dt

def decide_dt(d: Domain, fl: Fluid, prm: Params) -> float:
    """src/decide_dt.c:32-160."""
    small = 1.0e-8
    nx = d.nx
    dt = 1.0
    ux = V(d, fl.ux, 2, nx)
    dt = min(dt, float(np.min(M(d.hxxf, 2, nx) / (np.abs(ux) + small))))
    uy = V(d, fl.uy, 1, nx)
    dt = min(dt, float(np.min(M(d.hyxc, 1, nx) / (np.abs(uy) + small))))
    uz = V(d, fl.uz, 1, nx)
    dt = min(dt, float(np.min(d.hz / (np.abs(uz) + small))))
    dt *= prm.coef_dt_adv
    diffusivity = max(1.0 / fl.Re, 1.0 / fl.Re / fl.Pr)
    sizes = (float(np.min(d.hxxc)), d.hyxc[1], d.hz)
    for dim in range(3):
        dt_dif = prm.coef_dt_dif / diffusivity * 0.5 / 3 * sizes[dim] ** 2
        if not prm.implicit[dim]:
            dt = min(dt, dt_dif)
    return dt


# ---------------------------------------------------------------- tensors

def compute_tensors(d: Domain, fl: Fluid):
    """l_ij arrays with their y/z halos (src/fluid/predict/l*.c)."""
    nx = d.nx
    T = {}
    ux, uy, uz = fl.ux, fl.uy, fl.uz
    a = full(d)   # lxx, i=1..nx   lxx.c:28-34
    a[1:-1, 1:-1, 1:nx + 1] = 1.0 / M(d.hxxc, 1, nx) * (-V(d, ux, 1, nx) + V(d, ux, 1, nx, 1))
    T["lxx"] = a
    a = full(d)   # lxy, i=1..nx+1 lxy.c:28-34
    a[1:-1, 1:-1, 1:nx + 2] = 1.0 / M(d.hxxf, 1, nx + 1) * (-V(d, uy, 1, nx + 1, -1) + V(d, uy, 1, nx + 1))
    T["lxy"] = a
    a = full(d)   # lxz lxz.c:19-27
    a[1:-1, 1:-1, 1:nx + 2] = 1.0 / M(d.hxxf, 1, nx + 1) * (-V(d, uz, 1, nx + 1, -1) + V(d, uz, 1, nx + 1))
    T["lxz"] = a
    a = full(d)   # lyx0 lyx.c:33-39
    a[1:-1, 1:-1, 1:nx + 2] = 1.0 / M(d.hyxf, 1, nx + 1) * (-V(d, ux, 1, nx + 1, 0, -1) + V(d, ux, 1, nx + 1))
    T["lyx0"] = a
    a = full(d)   # lyx1 lyx.c:64-83
    hx_xm = M(d.hxxc, 1, nx + 1, -1)
    hx_xp = M(d.hxxc, 1, nx + 1)
    jd_xm = M(d.jdxc, 1, nx + 1, -1)
    jd_x0 = M(d.jdxf, 1, nx + 1)
    jd_xp = M(d.jdxc, 1, nx + 1)
    djdhx = -(jd_xm / hx_xm) + jd_xp / hx_xp
    wm = np.full(nx + 1, 0.5)
    wm[0] = 0.0
    wp = np.full(nx + 1, 0.5)
    wp[-1] = 0.0
    a[1:-1, 1:-1, 1:nx + 2] = -1.0 / jd_x0 * djdhx * (wm * V(d, uy, 1, nx + 1, -1) + wp * V(d, uy, 1, nx + 1))
    T["lyx1"] = a
    a = full(d)   # lyy0 lyy.c:33-39
    a[1:-1, 1:-1, 1:nx + 1] = 1.0 / M(d.hyxc, 1, nx) * (-V(d, uy, 1, nx) + V(d, uy, 1, nx, 0, 1))
    T["lyy0"] = a
    a = full(d)   # lyy1 lyy.c:64-83
    hx_xm = M(d.hxxf, 1, nx)
    hx_xp = M(d.hxxf, 1, nx, 1)
    jd_xm = M(d.jdxf, 1, nx)
    jd_x0 = M(d.jdxc, 1, nx)
    jd_xp = M(d.jdxf, 1, nx, 1)
    djdhx = -(jd_xm / hx_xm) + jd_xp / hx_xp
    a[1:-1, 1:-1, 1:nx + 1] = 1.0 / jd_x0 * djdhx * (0.5 * V(d, ux, 1, nx) + 0.5 * V(d, ux, 1, nx, 1))
    T["lyy1"] = a
    a = full(d)   # lyz lyz.c:19-27
    a[1:-1, 1:-1, 1:nx + 1] = 1.0 / M(d.hyxc, 1, nx) * (-V(d, uz, 1, nx, 0, -1) + V(d, uz, 1, nx))
    T["lyz"] = a
    a = full(d)   # lzx lzx.c
    a[1:-1, 1:-1, 1:nx + 2] = 1.0 / d.hz * (-V(d, ux, 1, nx + 1, 0, 0, -1) + V(d, ux, 1, nx + 1))
    T["lzx"] = a
    a = full(d)   # lzy
    a[1:-1, 1:-1, 1:nx + 1] = 1.0 / d.hz * (-V(d, uy, 1, nx, 0, 0, -1) + V(d, uy, 1, nx))
    T["lzy"] = a
    a = full(d)   # lzz
    a[1:-1, 1:-1, 1:nx + 1] = 1.0 / d.hz * (-V(d, uz, 1, nx) + V(d, uz, 1, nx, 0, 0, 1))
    T["lzz"] = a
    for a in T.values():
        halo_yz(a)
    fl.tensors = T
    return T


# ---------------------------------------------------------------- RHS

def laplacians(d: Domain, var: str):
    """(l, c, u) per radial index for x and y, scalars for z; lazily built
    tables in ux.c:34-81, uy.c:34-82, uz.c:29-78, t.c:29-78."""
    nx = d.nx
    if var == "ux":
        i = np.arange(2, nx + 1)
        lx = 1.0 / d.jdxf[i] * d.jdxc[i - 1] / d.hxxc[i - 1] / d.hxxc[i - 1]
        ux_ = 1.0 / d.jdxf[i] * d.jdxc[i] / d.hxxc[i] / d.hxxc[i]
        ly = 1.0 / d.hyxf[i] / d.hyxf[i]
    else:
        i = np.arange(1, nx + 1)
        lx = 1.0 / d.jdxc[i] * d.jdxf[i] / d.hxxf[i] / d.hxxf[i]
        ux_ = 1.0 / d.jdxc[i] * d.jdxf[i + 1] / d.hxxf[i + 1] / d.hxxf[i + 1]
        ly = 1.0 / d.hyxc[i] / d.hyxc[i]
    lapx = (lx, -lx - ux_, ux_)
    lapy = (ly, -ly - ly, ly)
    lz = 1.0 / d.hz / d.hz
    lapz = (lz, -lz - lz, lz)
    return lapx, lapy, lapz


def rhs_ux(d: Domain, fl: Fluid, prm: Params, srca, srcg):
    """compute_rhs_ux, src/fluid/predict/ux.c:92-439."""
    nx = d.nx
    lo, hi = 2, nx
    ux, uy, uz, p = fl.ux, fl.uy, fl.uz, fl.p
    T = fl.tensors
    X = lambda a, di=0, dj=0, dk=0: V(d, a, lo, hi, di, dj, dk)
    m = lambda arr, di=0: M(arr, lo, hi, di)
    nu = 1.0 / fl.Re
    lapx, lapy, lapz = laplacians(d, "ux")
    # advection_x :92-121
    hx_xm, hx_x0, hx_xp = m(d.hxxf, -1), m(d.hxxf), m(d.hxxf, 1)
    jd_xm, jd_x0, jd_xp = m(d.jdxf, -1), m(d.jdxf), m(d.jdxf, 1)
    ux_xm = 0.5 * jd_xm / hx_xm * X(ux, -1) + 0.5 * jd_x0 / hx_x0 * X(ux)
    ux_xp = 0.5 * jd_x0 / hx_x0 * X(ux) + 0.5 * jd_xp / hx_xp * X(ux, 1)
    l = -0.5 * ux_xm
    u = 0.5 * ux_xp
    c = -l - u
    srca -= 1.0 / jd_x0 * (l * X(ux, -1) + c * X(ux) + u * X(ux, 1))
    # advection_y :123-155
    hy_xm, hy_xp = m(d.hyxc, -1), m(d.hyxc)
    jd_xm, jd_x0, jd_xp = m(d.jdxc, -1), m(d.jdxf), m(d.jdxc)
    uy_ym = 0.5 * jd_xm / hy_xm * X(uy, -1) + 0.5 * jd_xp / hy_xp * X(uy)
    uy_yp = 0.5 * jd_xm / hy_xm * X(uy, -1, 1) + 0.5 * jd_xp / hy_xp * X(uy, 0, 1)
    l = -0.5 * uy_ym
    u = 0.5 * uy_yp
    c = -l - u
    srca -= 1.0 / jd_x0 * (l * X(ux, 0, -1) + c * X(ux) + u * X(ux, 0, 1))
    # advection_z :157-186
    uz_zm = 0.5 * jd_xm / d.hz * X(uz, -1) + 0.5 * jd_xp / d.hz * X(uz)
    uz_zp = 0.5 * jd_xm / d.hz * X(uz, -1, 0, 1) + 0.5 * jd_xp / d.hz * X(uz, 0, 0, 1)
    l = -0.5 * uz_zm
    u = 0.5 * uz_zp
    c = -l - u
    srca -= 1.0 / jd_x0 * (l * X(ux, 0, 0, -1) + c * X(ux) + u * X(ux, 0, 0, 1))
    # advection_1 (centrifugal) :194-226
    hx_xm, hx_x0, hx_xp = m(d.hxxf, -1), m(d.hxxf), m(d.hxxf, 1)
    jd_xm, jd_x0, jd_xp = m(d.jdxf, -1), m(d.jdxf), m(d.jdxf, 1)
    djdhx_xm = -(jd_xm / hx_xm) + jd_x0 / hx_x0
    djdhx_xp = -(jd_x0 / hx_x0) + jd_xp / hx_xp
    uy_xm = 0.5 * X(uy, -1) + 0.5 * X(uy, -1, 1)
    uy_xp = 0.5 * X(uy) + 0.5 * X(uy, 0, 1)
    srca += 1.0 / jd_x0 * (0.5 * djdhx_xm * uy_xm * uy_xm + 0.5 * djdhx_xp * uy_xp * uy_xp)
    # diffusion_x :228-245
    tgt = srcg if prm.implicit[0] else srca
    tgt += 2.0 * nu * (lapx[0] * X(ux, -1) + lapx[1] * X(ux) + lapx[2] * X(ux, 1))
    # diffusion_y0 :247-264
    tgt = srcg if prm.implicit[1] else srca
    tgt += nu * (lapy[0] * X(ux, 0, -1) + lapy[1] * X(ux) + lapy[2] * X(ux, 0, 1))
    # diffusion_y1 :266-290
    hy = m(d.hyxf)
    jd = m(d.jdxf)
    srca += nu / jd * (-(jd / hy) * (X(T["lyx1"]) + X(T["lxy"]))
                       + jd / hy * (X(T["lyx1"], 0, 1) + X(T["lxy"], 0, 1)))
    # diffusion_z0 :292-309
    tgt = srcg if prm.implicit[2] else srca
    tgt += nu * (lapz[0] * X(ux, 0, 0, -1) + lapz[1] * X(ux) + lapz[2] * X(ux, 0, 0, 1))
    # diffusion_z1 :311-332
    srca += nu / jd * (-(jd / d.hz) * X(T["lxz"]) + jd / d.hz * X(T["lxz"], 0, 0, 1))
    # diffusion_a :344-375
    hx_xm, hx_x0, hx_xp = m(d.hxxf, -1), m(d.hxxf), m(d.hxxf, 1)
    jd_xm, jd_x0, jd_xp = m(d.jdxf, -1), m(d.jdxf), m(d.jdxf, 1)
    djdhx_xm = -(jd_xm / hx_xm) + jd_x0 / hx_x0
    djdhx_xp = -(jd_x0 / hx_x0) + jd_xp / hx_xp
    lyy_xm = X(T["lyy0"], -1) + X(T["lyy1"], -1)
    lyy_xp = X(T["lyy0"]) + X(T["lyy1"])
    srca -= 2.0 * nu / jd_x0 * (0.5 * djdhx_xm * lyy_xm + 0.5 * djdhx_xp * lyy_xp)
    # pressure :377-394
    srcg -= 1.0 / m(d.hxxf) * (-X(p, -1) + X(p))


def rhs_uy(d: Domain, fl: Fluid, prm: Params, srca, srcg):
    """compute_rhs_uy, src/fluid/predict/uy.c:93-465."""
    nx = d.nx
    lo, hi = 1, nx
    ux, uy, uz, p = fl.ux, fl.uy, fl.uz, fl.p
    T = fl.tensors
    X = lambda a, di=0, dj=0, dk=0: V(d, a, lo, hi, di, dj, dk)
    m = lambda arr, di=0: M(arr, lo, hi, di)
    nu = 1.0 / fl.Re
    lapx, lapy, lapz = laplacians(d, "uy")
    # advection_x :93-123
    hx_xm, hx_xp = m(d.hxxf), m(d.hxxf, 1)
    jd_xm, jd_x0, jd_xp = m(d.jdxf), m(d.jdxc), m(d.jdxf, 1)
    ux_xm = 0.5 * jd_xm / hx_xm * X(ux, 0, -1) + 0.5 * jd_xm / hx_xm * X(ux)
    ux_xp = 0.5 * jd_xp / hx_xp * X(ux, 1, -1) + 0.5 * jd_xp / hx_xp * X(ux, 1)
    l = -0.5 * ux_xm
    u = 0.5 * ux_xp
    c = -l - u
    srca -= 1.0 / jd_x0 * (l * X(uy, -1) + c * X(uy) + u * X(uy, 1))
    # advection_y :125-151
    jd = m(d.jdxc)
    hy = m(d.hyxc)
    uy_ym = 0.5 * jd / hy * X(uy, 0, -1) + 0.5 * jd / hy * X(uy)
    uy_yp = 0.5 * jd / hy * X(uy) + 0.5 * jd / hy * X(uy, 0, 1)
    l = -0.5 * uy_ym
    u = 0.5 * uy_yp
    c = -l - u
    srca -= 1.0 / jd * (l * X(uy, 0, -1) + c * X(uy) + u * X(uy, 0, 1))
    # advection_z :153-180
    uz_zm = 0.5 * jd / d.hz * X(uz, 0, -1) + 0.5 * jd / d.hz * X(uz)
    uz_zp = 0.5 * jd / d.hz * X(uz, 0, -1, 1) + 0.5 * jd / d.hz * X(uz, 0, 0, 1)
    l = -0.5 * uz_zm
    u = 0.5 * uz_zp
    c = -l - u
    srca -= 1.0 / jd * (l * X(uy, 0, 0, -1) + c * X(uy) + u * X(uy, 0, 0, 1))
    # advection_1 (Coriolis-type) :188-223
    hx_xm, hx_xp = m(d.hxxf), m(d.hxxf, 1)
    jd_xm, jd_x0, jd_xp = m(d.jdxf), m(d.jdxc), m(d.jdxf, 1)
    djdhx = -(jd_xm / hx_xm) + jd_xp / hx_xp
    uy_ym = 0.5 * X(uy, 0, -1) + 0.5 * X(uy)
    uy_yp = 0.5 * X(uy) + 0.5 * X(uy, 0, 1)
    ux_ym = 0.5 * X(ux, 0, -1) + 0.5 * X(ux, 1, -1)
    ux_yp = 0.5 * X(ux) + 0.5 * X(ux, 1)
    srca -= 1.0 / jd_x0 * (0.5 * djdhx * uy_ym * ux_ym + 0.5 * djdhx * uy_yp * ux_yp)
    # diffusion_x0
    tgt = srcg if prm.implicit[0] else srca
    tgt += nu * (lapx[0] * X(uy, -1) + lapx[1] * X(uy) + lapx[2] * X(uy, 1))
    # diffusion_x1
    lyx_xm = X(T["lyx0"]) + X(T["lyx1"])
    lyx_xp = X(T["lyx0"], 1) + X(T["lyx1"], 1)
    srca += nu / jd_x0 * (-(jd_xm / hx_xm) * lyx_xm + jd_xp / hx_xp * lyx_xp)
    # diffusion_y0
    tgt = srcg if prm.implicit[1] else srca
    tgt += 2.0 * nu * (lapy[0] * X(uy, 0, -1) + lapy[1] * X(uy) + lapy[2] * X(uy, 0, 1))
    # diffusion_y1
    srca += 2.0 * nu / jd * (-(jd / hy) * X(T["lyy1"], 0, -1) + jd / hy * X(T["lyy1"]))
    # diffusion_z0
    tgt = srcg if prm.implicit[2] else srca
    tgt += nu * (lapz[0] * X(uy, 0, 0, -1) + lapz[1] * X(uy) + lapz[2] * X(uy, 0, 0, 1))
    # diffusion_z1
    srca += nu / jd * (-(jd / d.hz) * X(T["lyz"]) + jd / d.hz * X(T["lyz"], 0, 0, 1))
    # diffusion_a :367-400
    hx_xm, hx_x0, hx_xp = m(d.hxxc, -1), m(d.hxxc), m(d.hxxc, 1)
    jd_xm, jd_x0, jd_xp = m(d.jdxc, -1), m(d.jdxc), m(d.jdxc, 1)
    djdhx_xm = -(jd_xm / hx_xm) + jd_x0 / hx_x0
    djdhx_xp = -(jd_x0 / hx_x0) + jd_xp / hx_xp
    lyx_xm = X(T["lyx0"]) + X(T["lyx1"])
    lyx_xp = X(T["lyx0"], 1) + X(T["lyx1"], 1)
    lxy_xm = X(T["lxy"])
    lxy_xp = X(T["lxy"], 1)
    srca += nu / jd_x0 * (0.5 * djdhx_xm * (lyx_xm + lxy_xm) + 0.5 * djdhx_xp * (lyx_xp + lxy_xp))
    # pressure
    srcg -= 1.0 / m(d.hyxc) * (-X(p, 0, -1) + X(p))


def rhs_uz(d: Domain, fl: Fluid, prm: Params, srca, srcg):
    """compute_rhs_uz, src/fluid/predict/uz.c:88-359."""
    nx = d.nx
    lo, hi = 1, nx
    ux, uy, uz, p = fl.ux, fl.uy, fl.uz, fl.p
    T = fl.tensors
    X = lambda a, di=0, dj=0, dk=0: V(d, a, lo, hi, di, dj, dk)
    m = lambda arr, di=0: M(arr, lo, hi, di)
    nu = 1.0 / fl.Re
    lapx, lapy, lapz = laplacians(d, "uz")
    # advection_x
    hx_xm, hx_xp = m(d.hxxf), m(d.hxxf, 1)
    jd_xm, jd_x0, jd_xp = m(d.jdxf), m(d.jdxc), m(d.jdxf, 1)
    ux_xm = 0.5 * jd_xm / hx_xm * X(ux, 0, 0, -1) + 0.5 * jd_xm / hx_xm * X(ux)
    ux_xp = 0.5 * jd_xp / hx_xp * X(ux, 1, 0, -1) + 0.5 * jd_xp / hx_xp * X(ux, 1)
    l = -0.5 * ux_xm
    u = 0.5 * ux_xp
    c = -l - u
    srca -= 1.0 / jd_x0 * (l * X(uz, -1) + c * X(uz) + u * X(uz, 1))
    # advection_y
    hy = m(d.hyxc)
    jd = m(d.jdxc)
    uy_ym = 0.5 * jd / hy * X(uy, 0, 0, -1) + 0.5 * jd / hy * X(uy)
    uy_yp = 0.5 * jd / hy * X(uy, 0, 1, -1) + 0.5 * jd / hy * X(uy, 0, 1)
    l = -0.5 * uy_ym
    u = 0.5 * uy_yp
    c = -l - u
    srca -= 1.0 / jd * (l * X(uz, 0, -1) + c * X(uz) + u * X(uz, 0, 1))
    # advection_z
    uz_zm = 0.5 * jd / d.hz * X(uz, 0, 0, -1) + 0.5 * jd / d.hz * X(uz)
    uz_zp = 0.5 * jd / d.hz * X(uz) + 0.5 * jd / d.hz * X(uz, 0, 0, 1)
    l = -0.5 * uz_zm
    u = 0.5 * uz_zp
    c = -l - u
    srca -= 1.0 / jd * (l * X(uz, 0, 0, -1) + c * X(uz) + u * X(uz, 0, 0, 1))
    # diffusion_x0
    tgt = srcg if prm.implicit[0] else srca
    tgt += nu * (lapx[0] * X(uz, -1) + lapx[1] * X(uz) + lapx[2] * X(uz, 1))
    # diffusion_x1
    srca += nu / jd_x0 * (-(jd_xm / hx_xm) * X(T["lzx"]) + jd_xp / hx_xp * X(T["lzx"], 1))
    # diffusion_y0
    tgt = srcg if prm.implicit[1] else srca
    tgt += nu * (lapy[0] * X(uz, 0, -1) + lapy[1] * X(uz) + lapy[2] * X(uz, 0, 1))
    # diffusion_y1
    srca += nu / jd * (-(jd / hy) * X(T["lzy"]) + jd / hy * X(T["lzy"], 0, 1))
    # diffusion_z
    tgt = srcg if prm.implicit[2] else srca
    tgt += 2.0 * nu * (lapz[0] * X(uz, 0, 0, -1) + lapz[1] * X(uz) + lapz[2] * X(uz, 0, 0, 1))
    # pressure
    srcg -= 1.0 / d.hz * (-X(p, 0, 0, -1) + X(p))


def rhs_t(d: Domain, fl: Fluid, prm: Params, srca, srcg):
    """compute_rhs_t, src/fluid/predict/t.c:88-272."""
    nx = d.nx
    lo, hi = 1, nx
    ux, uy, uz, t = fl.ux, fl.uy, fl.uz, fl.t
    X = lambda a, di=0, dj=0, dk=0: V(d, a, lo, hi, di, dj, dk)
    m = lambda arr, di=0: M(arr, lo, hi, di)
    kappa = 1.0 / fl.Re / fl.Pr
    lapx, lapy, lapz = laplacians(d, "t")
    hx_xm, hx_xp = m(d.hxxf), m(d.hxxf, 1)
    jd_xm, jd_x0, jd_xp = m(d.jdxf), m(d.jdxc), m(d.jdxf, 1)
    ux_xm = jd_xm / hx_xm * X(ux)
    ux_xp = jd_xp / hx_xp * X(ux, 1)
    l = -0.5 * ux_xm
    u = 0.5 * ux_xp
    c = -l - u
    srca -= 1.0 / jd_x0 * (l * X(t, -1) + c * X(t) + u * X(t, 1))
    jd = m(d.jdxc)
    hy = m(d.hyxc)
    uy_ym = jd / hy * X(uy)
    uy_yp = jd / hy * X(uy, 0, 1)
    l = -0.5 * uy_ym
    u = 0.5 * uy_yp
    c = -l - u
    srca -= 1.0 / jd * (l * X(t, 0, -1) + c * X(t) + u * X(t, 0, 1))
    uz_zm = jd / d.hz * X(uz)
    uz_zp = jd / d.hz * X(uz, 0, 0, 1)
    l = -0.5 * uz_zm
    u = 0.5 * uz_zp
    c = -l - u
    srca -= 1.0 / jd * (l * X(t, 0, 0, -1) + c * X(t) + u * X(t, 0, 0, 1))
    tgt = srcg if prm.implicit[0] else srca
    tgt += kappa * (lapx[0] * X(t, -1) + lapx[1] * X(t) + lapx[2] * X(t, 1))
    tgt = srcg if prm.implicit[1] else srca
    tgt += kappa * (lapy[0] * X(t, 0, -1) + lapy[1] * X(t) + lapy[2] * X(t, 0, 1))
    tgt = srcg if prm.implicit[2] else srca
    tgt += kappa * (lapz[0] * X(t, 0, 0, -1) + lapz[1] * X(t) + lapz[2] * X(t, 0, 0, 1))


# ---------------------------------------------------------------- update

# which direction carries the doubled prefactor per variable:
# ux-x ux.c:502, uy-y uy.c:541, uz-z uz.c:451, t-y t.c:348
DOUBLED = {"ux": 0, "uy": 1, "uz": 2, "t": 1}


def implicit_solves(d: Domain, var: str, delta, prefactor, prm: Params):
    """solve_in_x / _y / _z (src/fluid/predict/linear_system.c:6-103) on the
    packed delta array (nz, ny, nI)."""
    lapx, lapy, lapz = laplacians(d, var)
    f = lambda dim: (2.0 if DOUBLED[var] == dim else 1.0) * prefactor
    if prm.implicit[0]:
        pf = f(0)
        l = -pf * lapx[0]
        c = 1.0 - pf * lapx[1]
        u = -pf * lapx[2]
        q = np.moveaxis(delta, 2, 0)
        gtsv(l, c, u, q)
    if prm.implicit[1]:
        pf = f(1)
        n = d.ny
        l = np.broadcast_to(-pf * lapy[0], (n,) + lapy[0].shape)
        c = np.broadcast_to(1.0 - pf * lapy[1], (n,) + lapy[1].shape)
        u = np.broadcast_to(-pf * lapy[2], (n,) + lapy[2].shape)
        q = np.moveaxis(delta, 1, 0)     # (ny, nz, nI); coefficients per i
        tdm_periodic(l[:, None, :], c[:, None, :], u[:, None, :], q)
    if prm.implicit[2]:
        pf = f(2)
        n = d.nz
        l = np.full(n, -pf * lapz[0])
        c = np.full(n, 1.0 - pf * lapz[1])
        u = np.full(n, -pf * lapz[2])
        tdm_periodic(l, c, u, delta)     # axis 0 is k


def predict_field(d: Domain, rkstep: int, dt: float, fl: Fluid, prm: Params):
    """fluid_predict_field (src/fluid/predict/main.c:35-110)."""
    # reset_srcs: alpha <-> beta, zero the new alpha and gamma (main.c:8-25)
    srcg = {}
    for v in fl.src:
        a, b = fl.src[v]
        fl.src[v] = [b, a]
        fl.src[v][0][...] = 0.0
        srcg[v] = np.zeros_like(a)
    compute_tensors(d, fl)
    rhs_ux(d, fl, prm, fl.src["ux"][0], srcg["ux"])
    rhs_uy(d, fl, prm, fl.src["uy"][0], srcg["uy"])
    rhs_uz(d, fl, prm, fl.src["uz"][0], srcg["uz"])
    rhs_t(d, fl, prm, fl.src["t"][0], srcg["t"])
    ca, cb, cg = RK_A[rkstep], RK_B[rkstep], RK_G[rkstep]
    for v in ("ux", "uy", "uz", "t"):
        delta = ca * dt * fl.src[v][0] + cb * dt * fl.src[v][1] + cg * dt * srcg[v]
        diff = 1.0 / fl.Re if v != "t" else 1.0 / fl.Re / fl.Pr
        implicit_solves(d, v, delta, 0.5 * RK_G[rkstep] * dt * diff, prm)
        arr = getattr(fl, v)
        lo = 2 if v == "ux" else 1
        V(d, arr, lo, d.nx)[...] += delta
    bc_ux(d, fl.ux)
    bc_uy(d, fl.uy, prm)
    bc_uz(d, fl.uz)
    bc_t(d, fl.t, prm)
    return srcg


# ---------------------------------------------------------------- Poisson

def divergence(d: Domain, ux, uy, uz):
    """div(u) at cell centres, compute_potential.c:382-425 (without scaling)."""
    nx = d.nx
    X = lambda a, di=0, dj=0, dk=0: V(d, a, 1, nx, di, dj, dk)
    m = lambda arr, di=0: M(arr, 1, nx, di)
    hx_xm, hx_xp, hy = m(d.hxxf), m(d.hxxf, 1), m(d.hyxc)
    jd_xm, jd_x0, jd_xp = m(d.jdxf), m(d.jdxc), m(d.jdxf, 1)
    return 1.0 / jd_x0 * (
        -(jd_xm / hx_xm) * X(ux) + jd_xp / hx_xp * X(ux, 1)
        - jd_x0 / hy * X(uy) + jd_x0 / hy * X(uy, 0, 1)
        - jd_x0 / d.hz * X(uz) + jd_x0 / d.hz * X(uz, 0, 0, 1))


def poisson_coefficients(d: Domain):
    """TDM l/u (compute_potential.c:173-211) and eigenvalues (:311-349)."""
    nx, ny, nz = d.nx, d.ny, d.nz
    i = np.arange(1, nx + 1)
    l = 1.0 / d.jdxc[i] * d.jdxf[i] / d.hxxf[i] / d.hxxf[i]
    u = 1.0 / d.jdxc[i] * d.jdxf[i + 1] / d.hxxf[i + 1] / d.hxxf[i + 1]
    pi = 3.14159265358979324
    ey = -4.0 * np.sin(pi * np.arange(ny // 2 + 1) / ny) ** 2
    ez = -4.0 * np.sin(pi * np.arange(nz) / nz) ** 2
    return l, u, ey, ez


def compute_potential(d: Domain, rkstep: int, dt: float, fl: Fluid, gauge: str = "pin"):
    """fluid_compute_potential (src/fluid/compute_potential.c:499-583).

    gauge="pin": the singular (0, 0) mode gets its last unknown set to zero
    (a fixed additive constant); gauge="reference": the reference's
    |pivot| <= DBL_EPSILON test (tdm.c:38-44) decides, which in practice
    leaves an arbitrary constant in psi."""
    nx, ny, nz = d.nx, d.ny, d.nz
    norm = 1.0 * ny * nz
    prefactor = 1.0 / (RK_G[rkstep] * dt) / norm
    rhs = prefactor * divergence(d, fl.ux, fl.uy, fl.uz)       # (nz, ny, nx)
    spec = np.fft.rfft(rhs, axis=1)                             # y r2c
    spec = np.fft.fft(spec, axis=0)                             # z forward
    l, u, ey, ez = poisson_coefficients(d)
    hyxc = d.hyxc[1:nx + 1]
    c = (-l - u)[None, None, :] + ey[None, :, None] / hyxc / hyxc + ez[:, None, None] / d.hz / d.hz
    c = np.array(c)
    c[:, :, 0] += l[0]
    c[:, :, nx - 1] += u[nx - 1]
    q = np.moveaxis(spec, 2, 0)                                 # (nx, nz, nyh)
    cc = np.moveaxis(c, 2, 0)
    if gauge == "pin":
        # solve the (0,0) mode with its last unknown fixed to zero
        c00 = cc[:, 0, 0].copy()
        q00 = q[:, 0, 0].copy()
        cc[nx - 1, 0, 0] = 1.0
        gtsv(l[:, None, None], cc, u[:, None, None], q)
        sub = q00[:nx - 1].copy()
        gtsv(l[:nx - 1], c00[:nx - 1], u[:nx - 1], sub)
        q[:nx - 1, 0, 0] = sub
        q[nx - 1, 0, 0] = 0.0
    else:
        gtsv(l[:, None, None], cc, u[:, None, None], q)
    spec = np.moveaxis(q, 0, 2)
    spec = np.fft.ifft(spec, axis=0) * nz                       # z backward, unnormalised
    out = np.fft.irfft(spec, n=ny, axis=1) * ny                 # y c2r, unnormalised
    V(d, fl.psi, 1, nx)[...] = out
    bc_psi(d, fl.psi)


def correct_velocity(d: Domain, rkstep: int, dt: float, fl: Fluid, prm: Params):
    """fluid_correct_velocity (src/fluid/correct/*.c)."""
    nx = d.nx
    pf = RK_G[rkstep] * dt
    psi = fl.psi
    V(d, fl.ux, 2, nx)[...] -= pf / M(d.hxxf, 2, nx) * (-V(d, psi, 2, nx, -1) + V(d, psi, 2, nx))
    bc_ux(d, fl.ux)
    V(d, fl.uy, 1, nx)[...] -= pf / M(d.hyxc, 1, nx) * (-V(d, psi, 1, nx, 0, -1) + V(d, psi, 1, nx))
    bc_uy(d, fl.uy, prm)
    V(d, fl.uz, 1, nx)[...] -= pf / d.hz * (-V(d, psi, 1, nx, 0, 0, -1) + V(d, psi, 1, nx))
    bc_uz(d, fl.uz)


def update_pressure(d: Domain, rkstep: int, dt: float, fl: Fluid, prm: Params):
    """fluid_update_pressure (src/fluid/update_pressure.c:23-173)."""
    nx = d.nx
    P = V(d, fl.p, 1, nx)
    psi = fl.psi
    X = lambda di=0, dj=0, dk=0: V(d, psi, 1, nx, di, dj, dk)
    P += X()
    pf = 0.5 * RK_G[rkstep] * dt * (1.0 / fl.Re)
    if prm.implicit[0]:
        hx_xm, hx_xp = M(d.hxxf, 1, nx), M(d.hxxf, 1, nx, 1)
        jd_xm, jd_x0, jd_xp = M(d.jdxf, 1, nx), M(d.jdxc, 1, nx), M(d.jdxf, 1, nx, 1)
        l = jd_xm / hx_xm / hx_xm
        u = jd_xp / hx_xp / hx_xp
        c = -l - u
        P -= 2.0 * pf / jd_x0 * (l * X(-1) + c * X() + u * X(1))
    if prm.implicit[1]:
        hy, jd = M(d.hyxc, 1, nx), M(d.jdxc, 1, nx)
        l = jd / hy / hy
        u = jd / hy / hy
        c = -l - u
        P -= 2.0 * pf / jd * (l * X(0, -1) + c * X() + u * X(0, 1))
    if prm.implicit[2]:
        jd = M(d.jdxc, 1, nx)
        l = jd / d.hz / d.hz
        u = jd / d.hz / d.hz
        c = -l - u
        P -= 2.0 * pf / jd * (l * X(0, 0, -1) + c * X() + u * X(0, 0, 1))
    bc_p(d, fl.p)


def integrate(d: Domain, fl: Fluid, prm: Params, gauge: str = "pin") -> float:
    """integrate (src/integrate.c:9-35)."""
    dt = decide_dt(d, fl, prm)
    for rk in range(3):
        predict_field(d, rk, dt, fl, prm)
        compute_potential(d, rk, dt, fl, gauge=gauge)
        correct_velocity(d, rk, dt, fl, prm)
        update_pressure(d, rk, dt, fl, prm)
    return dt


# ---------------------------------------------------------------- logging

def diagnostics(d: Domain, fl: Fluid) -> dict:
    """src/logging/divergence.c:32-91, injection.c:31-103,
    dissipation.c:27-371, total_energy.c:22-93, from the current fields."""
    nx = d.nx
    T = compute_tensors(d, fl)
    out = {}
    out["divmax"] = float(np.max(np.abs(divergence(d, fl.ux, fl.uy, fl.uz))))
    nu = 1.0 / fl.Re
    kappa = 1.0 / fl.Re / fl.Pr
    j = slice(1, d.ny + 1)
    k = slice(1, d.nz + 1)
    tyx_m = T["lyx0"][k, j, 1] + T["lyx1"][k, j, 1] + T["lxy"][k, j, 1]
    tyx_p = T["lyx0"][k, j, nx + 1] + T["lyx1"][k, j, nx + 1] + T["lxy"][k, j, nx + 1]
    inj = (-d.jdxf[1] / d.hxxf[1] * fl.uy[k, j, 0] * tyx_m
           + d.jdxf[nx + 1] / d.hxxf[nx + 1] * fl.uy[k, j, nx + 1] * tyx_p)
    out["injection_u"] = nu * float(np.sum(inj))
    t = fl.t
    inj_t = (-d.jdxf[1] / d.hxxf[1] * t[k, j, 0] / d.hxxf[1] * (-t[k, j, 0] + t[k, j, 1])
             + d.jdxf[nx + 1] / d.hxxf[nx + 1] * t[k, j, nx + 1] / d.hxxf[nx + 1] * (-t[k, j, nx] + t[k, j, nx + 1]))
    out["injection_t"] = kappa * float(np.sum(inj_t))
    F = lambda a: V(d, a, 1, nx + 1)
    Cc = lambda a: V(d, a, 1, nx)
    jf = M(d.jdxf, 1, nx + 1)
    jc = M(d.jdxc, 1, nx)
    lyx = F(T["lyx0"]) + F(T["lyx1"])
    lxy = F(T["lxy"])
    lzx = F(T["lzx"])
    lxz = F(T["lxz"])
    lyy = Cc(T["lyy0"]) + Cc(T["lyy1"])
    dis = (np.sum(jc * Cc(T["lxx"]) * (Cc(T["lxx"]) + Cc(T["lxx"])))
           + np.sum(jf * lyx * (lyx + lxy)) + np.sum(jf * lzx * (lzx + lxz)) + np.sum(jf * lxy * (lxy + lyx))
           + np.sum(jc * lyy * (lyy + lyy)) + np.sum(jc * Cc(T["lzy"]) * (Cc(T["lzy"]) + Cc(T["lyz"])))
           + np.sum(jf * lxz * (lxz + lzx)) + np.sum(jc * Cc(T["lyz"]) * (Cc(T["lyz"]) + Cc(T["lzy"])))
           + np.sum(jc * Cc(T["lzz"]) * (Cc(T["lzz"]) + Cc(T["lzz"]))))
    out["dissipation_u"] = nu * float(dis)
    dtx = (-V(d, t, 1, nx + 1, -1) + V(d, t, 1, nx + 1)) / M(d.hxxf, 1, nx + 1)
    dty = (-V(d, t, 1, nx, 0, -1) + V(d, t, 1, nx)) / M(d.hyxc, 1, nx)
    dtz = (-V(d, t, 1, nx, 0, 0, -1) + V(d, t, 1, nx)) / d.hz
    out["dissipation_t"] = kappa * float(np.sum(jf * dtx ** 2) + np.sum(jc * dty ** 2) + np.sum(jc * dtz ** 2))
    out["energy_ux"] = float(np.sum(M(d.jdxf, 2, nx) * 0.5 * V(d, fl.ux, 2, nx) ** 2))
    out["energy_uy"] = float(np.sum(jc * 0.5 * V(d, fl.uy, 1, nx) ** 2))
    out["energy_uz"] = float(np.sum(jc * 0.5 * V(d, fl.uz, 1, nx) ** 2))
    out["energy_t"] = float(np.sum(jc * 0.5 * V(d, fl.t, 1, nx) ** 2))
    return out
