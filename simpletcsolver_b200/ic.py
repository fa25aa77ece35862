"""Seeded initial-condition generator with the reference's NPY schema.

The reference ships an unseeded generator (initial_condition/main.py:46-129:
clipped-Chebyshev radial grid, uniform noise in [0, 1)). This one writes the
same files with the same shapes and dtypes, so the reference and this library
load its output unchanged (src/main.c:46-52, src/domain.c:28-55,
src/fluid/init.c:98-110):

    step.npy  <u8 ()          time.npy    <f8 ()
    is_curved.npy |b1 ()      glsizes.npy <u8 (3,)    lengths.npy <f8 (3,)
    xf.npy  <f8 (nx+1,)       xc.npy      <f8 (nx+2,)
    ux.npy  <f8 (nz, ny, nx+1)
    uy.npy, uz.npy, p.npy, t.npy  <f8 (nz, ny, nx+2)

Differences from the reference generator, all deliberate:
  * the radial faces are tanh-clustered towards both walls
    (xf = xmin + lx/2 * (1 + tanh(beta*(2s-1)) / tanh(beta)), s = i/nx);
  * the azimuthal velocity starts from the laminar profile (circular Couette
    uy = A r + B/r when curved, linear plane Couette when planar), the scalar
    from a linear profile between the wall values;
  * noise is uniform in [-amp, amp) from numpy.random.default_rng(seed), drawn
    in the order ux, uy, uz, t.
"""
from __future__ import annotations

import dataclasses
import math
import os

import numpy as np


@dataclasses.dataclass(frozen=True)
class Case:
    """Geometry, grid, physics and initial field of one run."""
    is_curved: bool
    nx: int
    ny: int
    nz: int
    lx: float
    ly: float
    lz: float
    Re: float
    Pr: float = 1.0
    stretch: float = 1.5
    uy_xm: float = 1.0
    uy_xp: float = 0.0
    t_xm: float = 0.5
    t_xp: float = -0.5
    implicit: tuple = (True, False, False)
    noise_u: float = 0.05
    noise_t: float = 0.0
    seed: int = 0
    coef_dt_adv: float = 0.4
    coef_dt_dif: float = 1.0

    @property
    def xmin(self) -> float:
        return 1.0 if self.is_curved else 0.0

    @property
    def ncells(self) -> int:
        return self.nx * self.ny * self.nz


def taylor_couette(nx, ny, nz, Re, **kw) -> Case:
    """Curved channel of the Taylor-Couette workloads: inner radius 1, outer
    1.4, inner wall at speed 1, outer at rest, azimuthal span 2*pi/10, axial
    length 2.094, noise U(-0.05, 0.05) on all velocity components."""
    args = dict(is_curved=True, nx=nx, ny=ny, nz=nz, lx=0.4, ly=2.0 * math.pi / 10.0,
                lz=2.094, Re=Re, Pr=1.0, uy_xm=1.0, uy_xp=0.0, t_xm=0.5, t_xp=-0.5,
                implicit=(True, False, False), noise_u=0.05, noise_t=0.0)
    args.update(kw)
    return Case(**args)


def plane_couette(nx, ny, nz, Re, **kw) -> Case:
    """Planar channel workload: walls moving at -0.5 / +0.5, scalar 1 / 0 at
    the walls, implicit diffusion in all three directions, noise U(-0.01, 0.01)."""
    args = dict(is_curved=False, nx=nx, ny=ny, nz=nz, lx=1.0, ly=2.0, lz=1.0, Re=Re,
                Pr=1.0, uy_xm=-0.5, uy_xp=0.5, t_xm=1.0, t_xp=0.0,
                implicit=(True, True, True), noise_u=0.01, noise_t=0.01)
    args.update(kw)
    return Case(**args)


# the workloads, by what they are
TC_SMALL = taylor_couette(64, 128, 64, 3400.0)        # CPU-runnable Taylor-Couette
TC_LARGE = taylor_couette(256, 1024, 512, 1.0e4)      # the headline Taylor-Couette grid
PLANAR = plane_couette(192, 512, 256, 2000.0)         # planar channel with scalar
TC_COARSE = taylor_couette(64, 256, 128, 1.0e4)       # 4x-coarsened Taylor-Couette


def radial_grid(case: Case):
    """Cell faces xf (nx+1) and centres xc (nx+2, walls included as the
    first and last entries, as initial_condition/main.py:71-74 lays them out)."""
    s = np.arange(case.nx + 1, dtype=np.float64) / case.nx
    beta = case.stretch
    xf = 0.5 * case.lx * (1.0 + np.tanh(beta * (2.0 * s - 1.0)) / math.tanh(beta))
    xf[0] = 0.0
    xf[-1] = case.lx
    xc = np.concatenate(([0.0], 0.5 * (xf[:-1] + xf[1:]), [case.lx]))
    return xf + case.xmin, xc + case.xmin


def initial_fields(case: Case, xf=None, xc=None):
    """Return dict of ux, uy, uz, p, t arrays in NPY shape (nz, ny, nx+adds)."""
    if xf is None:
        xf, xc = radial_grid(case)
    nx, ny, nz = case.nx, case.ny, case.nz
    rng = np.random.default_rng(case.seed)
    ri, ro = case.xmin, case.xmin + case.lx
    if case.is_curved:
        ui, uo = case.uy_xm, case.uy_xp
        a = (uo * ro - ui * ri) / (ro * ro - ri * ri)
        b = (ui - a * ri) * ri
        uy_profile = a * xc + b / xc
    else:
        uy_profile = case.uy_xm + (case.uy_xp - case.uy_xm) * (xc - ri) / case.lx
    t_profile = case.t_xm + (case.t_xp - case.t_xm) * (xc - ri) / case.lx
    amp = case.noise_u
    ux = rng.uniform(-amp, amp, size=(nz, ny, nx + 1))
    uy = uy_profile[None, None, :] + rng.uniform(-amp, amp, size=(nz, ny, nx + 2))
    uz = rng.uniform(-amp, amp, size=(nz, ny, nx + 2))
    t = np.broadcast_to(t_profile, (nz, ny, nx + 2)).copy()
    if case.noise_t > 0.0:
        t += rng.uniform(-case.noise_t, case.noise_t, size=(nz, ny, nx + 2))
    p = np.zeros((nz, ny, nx + 2))
    # walls: impermeable, no-slip (the solver re-imposes these on load)
    ux[:, :, 0] = 0.0
    ux[:, :, -1] = 0.0
    return dict(ux=ux, uy=uy, uz=uz, p=p, t=t)


def write_domain(case: Case, dest: str, step: int = 0, time: float = 0.0) -> str:
    """The small files of an initial-condition directory (step, time and the
    domain: src/main.c:46-52, src/domain.c:28-55), without the fields."""
    os.makedirs(dest, exist_ok=True)
    xf, xc = radial_grid(case)
    np.save(os.path.join(dest, "step.npy"), np.array(step, dtype=np.uint64))
    np.save(os.path.join(dest, "time.npy"), np.array(time, dtype=np.float64))
    np.save(os.path.join(dest, "is_curved.npy"), np.array(case.is_curved, dtype=np.bool_))
    np.save(os.path.join(dest, "glsizes.npy"), np.array([case.nx, case.ny, case.nz], dtype=np.uint64))
    np.save(os.path.join(dest, "lengths.npy"), np.array([case.lx, case.ly, case.lz], dtype=np.float64))
    np.save(os.path.join(dest, "xf.npy"), xf)
    np.save(os.path.join(dest, "xc.npy"), xc)
    return dest


def write_ic(case: Case, dest: str, step: int = 0, time: float = 0.0) -> str:
    """Write an initial-condition directory that both solvers load."""
    write_domain(case, dest, step, time)
    xf, xc = radial_grid(case)
    for name, arr in initial_fields(case, xf, xc).items():
        np.save(os.path.join(dest, f"{name}.npy"), np.ascontiguousarray(arr, dtype=np.float64))
    return dest


def case_env(case: Case) -> dict:
    """Environment variables the reference reads at start-up (src/config.c)."""
    return {"Re": repr(case.Re), "Pr": repr(case.Pr),
            "coef_dt_adv": repr(case.coef_dt_adv), "coef_dt_dif": repr(case.coef_dt_dif)}
