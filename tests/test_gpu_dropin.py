"""The reference's own host program on the GPU library, and the device-side
logging and statistics against the reference's.

oracle/_ref/tcdropin is the reference's src/main.c with its logging/,
save.c, statistics.c, fileio.c, config.c, timer.c, memory.c and array.c,
compiled unmodified and linked against libtcgpu.so in place of the solver
sources (oracle/Makefile, target dropin). oracle/_ref/tcmain_tc is the same
program built entirely from the reference's sources. Both run the same
seeded case in their own working directories; the drop-in gets
TCGPU_SYNC_TENSORS=1 so that the host tensors its logging and statistics read
are those the reference leaves behind (src/fluid/predict/main.c:56-82).

Tolerances: logged quantities 1e-9 relative (the reference prints 16
significant digits), fields and statistics 1e-10 relative L2 after about 60
steps, divergence below 1e-12 in both runs.
"""
import math
import os
import subprocess

import numpy as np
import pytest

from simpletcsolver_b200 import ic
from simpletcsolver_b200.solver import Solver
from tests._helpers import REF_DIR, rel_l2

pytestmark = pytest.mark.gpu

CASE = ic.taylor_couette(16, 32, 16, 3400.0)
RUN_ENV = {"timemax": "0.5", "wtimemax": "600", "log_rate": "0.05", "save_rate": "0.25", "save_after": "0",
           "stat_rate": "0.05", "stat_after": "0.1"}
STAT_NAMES = ("ux1", "ux2", "uy1", "uy2", "uz1", "uz2", "adv", "dif")


def have(name):
    return os.path.exists(os.path.join(REF_DIR, name))


def run_program(exe, ic_dir, cwd, extra=None):
    for sub in ("log", "save", "stat"):
        os.makedirs(os.path.join(cwd, "output", sub), exist_ok=True)
    env = dict(os.environ, **ic.case_env(CASE), **RUN_ENV, **(extra or {}))
    r = subprocess.run([os.path.join(REF_DIR, exe), ic_dir], cwd=cwd, env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return os.path.join(cwd, "output")


def read_log(out, name):
    rows = [line.split() for line in open(os.path.join(out, "log", name + ".dat")) if line.strip()]
    return np.array([[float(v) for v in r] for r in rows])


def latest(out, sub):
    dirs = sorted(d for d in os.listdir(os.path.join(out, sub)))
    assert dirs, f"no {sub} directory written"
    return os.path.join(out, sub, dirs[-1])


@pytest.fixture(scope="module")
def reference_run(tmp_path_factory):
    if not have("tcmain_tc"):
        pytest.skip("reference build oracle/_ref absent")
    root = tmp_path_factory.mktemp("refmain")
    ic_dir = ic.write_ic(CASE, str(root / "ic"))
    return ic_dir, run_program("tcmain_tc", ic_dir, str(root / "cpu"))


def test_reference_main_runs_on_the_library(lib, reference_run, tmp_path):
    """Unmodified reference host program linked against libtcgpu.so: same
    logs, saves and statistics as the all-CPU reference program."""
    if not have("tcdropin"):
        pytest.skip("drop-in build oracle/_ref/tcdropin absent")
    ic_dir, cpu = reference_run
    gpu = run_program("tcdropin", ic_dir, str(tmp_path / "gpu"), {"TCGPU_SYNC_TENSORS": "1"})
    # progress: the same steps at the same times
    a = [line.split(",")[:3] for line in open(os.path.join(cpu, "log", "progress.dat"))]
    b = [line.split(",")[:3] for line in open(os.path.join(gpu, "log", "progress.dat"))]
    assert a == b and len(a) >= 8
    for name in ("injection", "dissipation", "total_energy"):
        x, y = read_log(cpu, name), read_log(gpu, name)
        assert x.shape == y.shape, name
        np.testing.assert_array_equal(x[:, 0], y[:, 0])
        np.testing.assert_allclose(y[:, 1:], x[:, 1:], rtol=1e-9, atol=0, err_msg=name)
    for out in (cpu, gpu):
        assert read_log(out, "divergence")[:, 1].max() < 1e-12
    # saves: same directories, same fields
    assert sorted(os.listdir(os.path.join(cpu, "save"))) == sorted(os.listdir(os.path.join(gpu, "save")))
    for d in os.listdir(os.path.join(cpu, "save")):
        for n in ("ux", "uy", "uz", "t"):
            x = np.load(os.path.join(cpu, "save", d, n + ".npy"))
            y = np.load(os.path.join(gpu, "save", d, n + ".npy"))
            assert rel_l2(y, x) < 1e-10, (d, n)
        for n in ("step", "glsizes", "xf", "xc"):
            np.testing.assert_array_equal(np.load(os.path.join(cpu, "save", d, n + ".npy")),
                                          np.load(os.path.join(gpu, "save", d, n + ".npy")), err_msg=n)
        # dt is the minimum of h / |u| over fields equal to round-off, so the
        # summed time may differ in its last bits
        assert float(np.load(os.path.join(gpu, "save", d, "time.npy"))) == pytest.approx(
            float(np.load(os.path.join(cpu, "save", d, "time.npy"))), rel=1e-13)
    # statistics collected by the reference's statistics.c from the library's host arrays
    sc, sg = latest(cpu, "stat"), latest(gpu, "stat")
    assert os.path.basename(sc) == os.path.basename(sg)
    assert int(np.load(os.path.join(sc, "num.npy"))) == int(np.load(os.path.join(sg, "num.npy"))) > 0
    for n in STAT_NAMES:
        assert rel_l2(np.load(os.path.join(sg, n + ".npy")), np.load(os.path.join(sc, n + ".npy"))) < 1e-10, n


def schedule(rate, after, time):
    """logging/main.c:21-24 and statistics.c:61-63: the first output time."""
    return rate * math.ceil(max(np.finfo(float).eps, max(time, after)) / rate)


def test_device_logging_and_statistics_follow_the_reference(lib, reference_run, tmp_path):
    """Resident steps with the reference main loop's schedule: the logged
    quantities (tcgpu_log_quantities, the reference's stale tensors) and the
    statistics accumulated on the device (tcgpu_statistics_*) against the
    all-CPU reference program's own logs and statistics directory."""
    ic_dir, cpu = reference_run
    s = Solver.from_ic(ic_dir, case=CASE, lib=lib)
    try:
        s.push()
        timemax = float(RUN_ENV["timemax"])
        log_rate, stat_rate = float(RUN_ENV["log_rate"]), float(RUN_ENV["stat_rate"])
        log_next = schedule(log_rate, 0.0, 0.0)
        stat_next = schedule(stat_rate, float(RUN_ENV["stat_after"]), 0.0)
        time, step, logs = 0.0, 0, []
        while True:                                   # src/main.c:87-118
            time += float(s.run(1)[0])
            step += 1
            if timemax < time:
                break
            if log_next < time:
                q = s.log_quantities()
                logs.append([q["injection_u"], q["injection_t"], q["dissipation_u"], q["dissipation_t"],
                             q["energy_ux"], q["energy_uy"], q["energy_uz"], q["energy_t"], q["divmax"]])
                log_next += log_rate
            if stat_next < time:
                s.stats_collect()
                stat_next += stat_rate
        logs = np.array(logs)
        inj, dis, ene = (read_log(cpu, n) for n in ("injection", "dissipation", "total_energy"))
        assert len(logs) == len(inj) >= 8
        np.testing.assert_allclose(logs[:, 0:2], inj[:, 1:3], rtol=1e-9, atol=0)
        np.testing.assert_allclose(logs[:, 2:4], dis[:, 1:3], rtol=1e-9, atol=0)
        np.testing.assert_allclose(logs[:, 4:8], ene[:, 1:5], rtol=1e-9, atol=0)
        assert logs[:, 8].max() < 1e-12
        num, arrays = s.stats()
        sc = latest(cpu, "stat")
        assert num == int(np.load(os.path.join(sc, "num.npy"))) > 0
        for n in STAT_NAMES:
            assert rel_l2(arrays[n], np.load(os.path.join(sc, n + ".npy"))) < 1e-10, n
        # the reference's statistics directory, written by the library
        out = str(tmp_path / "stat")
        s.stats_save(out)
        for n in STAT_NAMES + ("num", "glsizes", "xf", "xc"):
            a, b = np.load(os.path.join(out, n + ".npy")), np.load(os.path.join(sc, n + ".npy"))
            assert a.shape == b.shape and a.dtype == b.dtype, n
        # mean uy(r) profile = mean of uy1 over j, k and the samples
        prof = s.mean_uy()
        np.testing.assert_allclose(prof, arrays["uy1"].mean(axis=(0, 1)) / num, rtol=1e-12, atol=1e-15)
        s.stats_reset()
        assert s.stats()[0] == 0 and not s.stats()[1]["uy1"].any()
    finally:
        s.release()
