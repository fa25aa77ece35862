"""Shared helpers of the test suite: golden fixtures, oracle runs, comparisons."""
from __future__ import annotations

import json
import os

import numpy as np

from oracle import tc_numpy as tn
from simpletcsolver_b200 import ic

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def have_ref(build: str = "tc") -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"tcref_{build}"))


def load_golden(name: str):
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    meta = json.loads(str(z["meta"]))
    meta["case"]["implicit"] = tuple(meta["case"]["implicit"])
    case = ic.Case(**meta["case"])
    return z, meta, case


def params_of(case: ic.Case) -> tn.Params:
    return tn.Params(uy_xm=case.uy_xm, uy_xp=case.uy_xp, t_xm=case.t_xm, t_xp=case.t_xp,
                     implicit=tuple(case.implicit), coef_dt_adv=case.coef_dt_adv, coef_dt_dif=case.coef_dt_dif)


def oracle_from_golden(z, case):
    d = tn.make_domain(bool(z["ic_is_curved"]), z["ic_glsizes"], z["ic_lengths"], z["ic_xf"], z["ic_xc"])
    fields = {n: z["ic_" + n] for n in ("ux", "uy", "uz", "p", "t")}
    fl = tn.make_fluid(d, fields, case.Re, case.Pr, params_of(case))
    return d, fl


def write_ic_from_golden(z, dest: str) -> str:
    os.makedirs(dest, exist_ok=True)
    for n in ("ux", "uy", "uz", "p", "t", "xf", "xc", "glsizes", "lengths", "is_curved"):
        np.save(os.path.join(dest, n + ".npy"), z["ic_" + n])
    np.save(os.path.join(dest, "step.npy"), np.array(0, dtype=np.uint64))
    np.save(os.path.join(dest, "time.npy"), np.array(0.0))
    return dest


def oracle_layout(name: str, a):
    """Host / reference layout (ux rows of nx+1) -> oracle layout (nx+2)."""
    if name != "ux":
        return a
    out = np.zeros(a.shape[:2] + (a.shape[2] + 1,))
    out[:, :, 1:] = a
    return out


def rel_l2(a, b, interior=None):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def demean(a):
    """Remove the additive pressure gauge: subtract the mean of the interior."""
    return a - a[1:-1, 1:-1, 1:-1].mean()
