#!/usr/bin/env python
"""Throughput of SimpleTCSolver's RK3 time step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl tcgpu|reference]

Workload: the Taylor-Couette case at Re=1e4 on the 256x1024x512 grid (FP64),
seeded synthetic noisy circular-Couette initial field. One step = decide_dt +
three RK substeps of predict / Poisson / correct / pressure (src/integrate.c).

Metric: Mcell-steps/s = nx*ny*nz * steps / device seconds, summed over ranks.
  value     device time of K steps with the state resident in HBM (CUDA events
            on the library's stream, the step replayed as one CUDA graph)
  e2e       the same K steps through the reference entry point integrate()
            with host arrays: every step copies ux, uy, uz, p, t host->device
            and ux, uy, uz, p, t, psi back (page-locked host memory)
  roofline  the kernel with the largest share of the step: algorithmic bytes
            per launch / its mean launch time from events around each launch
Multi-GPU: the path does not shard (global FFTs, single-rank drop-in), so N GPUs
run N independent replicas ("scaling": "weak"); time = max over ranks.

--impl reference times the reference's own CPU code (oracle/_ref/tcref_tc,
built from the reference sources) on this host's cores: P single-rank
processes, each integrating a 64x128x64 sample of the same case, throughput
summed; rank 0 only.
"""
from __future__ import annotations

import argparse
import ctypes as C
import csv
import datetime
import io
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-steps/s on 1 B200 (plain FP64 vs chosen form); torque err vs FP64 fine"
UNIT = "Mcell-steps/s"
WORKLOAD = "taylor-couette 256x1024x512 Re=1e4 fp64"
SAMPLE_GRID = (64, 128, 64)

# algorithmic bytes per cell and launch (8-byte words): reads + writes each kernel must do
KERNELS = ["DTMIN", "DTFINAL", "FACTORS", "PREDICT", "APPLY", "YZSOLVE", "DIV_FFTY", "FFTZ_FWD", "TDM",
           "FFTZ_INV", "IFFTY", "CORRECT"]
BYTES_PER_CELL = {
    "DTMIN": 3 * 8,                            # ux, uy, uz
    # fused predict: 5 fields read, srcA_new + new ux, uy, uz, t written (104 B);
    # substeps 2 and 3 also read srcA_old (136 B)
    "PREDICT": (104.0 + 136.0 + 136.0) / 3.0,
    "DIV_FFTY": 3 * 8 + 8,                     # ux, uy, uz read; half-spectrum written
    "FFTZ_FWD": 16, "TDM": 16, "FFTZ_INV": 16,  # spectrum read + written
    "IFFTY": 8 + 8,                            # spectrum read, psi written
    "CORRECT": 9 * 8,                          # psi, ux, uy, uz, p read; ux, uy, uz, p written
}
MODEL_BYTES_PER_CELL_STEP = 912
# FP32-storage mode: ux, uy, uz, t, the source terms and the spectra in 4 bytes,
# p and psi in 8
BYTES_PER_CELL_FP32 = {
    "DTMIN": 3 * 4,
    # predict: ux, uy, uz, t (4 B) and p (8 B) read, 4 new sources + 4 fields
    # written (56 B); substeps 2 and 3 also read the old sources (72 B)
    "PREDICT": (56.0 + 72.0 + 72.0) / 3.0,
    "DIV_FFTY": 3 * 4 + 4,
    "FFTZ_FWD": 8, "TDM": 8, "FFTZ_INV": 8,
    "IFFTY": 4 + 8,
    "CORRECT": 8 + 12 + 8 + 12 + 8,            # psi, ux, uy, uz, p read; ux, uy, uz, p written
}
MODEL_BYTES_PER_CELL_STEP_FP32 = 500           # 200 (predict) + 3 x 100 (Poisson + correction)


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["tcgpu", "reference"], default="tcgpu")
    ap.add_argument("--grid", type=str, default="256x1024x512")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp32", action="store_true", help="skip the FP32-storage arm")
    ap.add_argument("--accuracy-steps", type=int, default=200,
                    help="steps of the FP32-storage vs FP64 accuracy runs (0: skip)")
    ap.add_argument("--no-closure", action="store_true", help="skip the learned-closure arm")
    ap.add_argument("--no-planar", action="store_true", help="skip the planar-channel workload")
    ap.add_argument("--closure-pairs", type=int, default=200, help="training pairs from the fine run")
    ap.add_argument("--closure-epochs", type=int, default=60)
    ap.add_argument("--closure-warm", type=int, default=200,
                    help="fine steps before the first pair (lets the initial noise decay)")
    ap.add_argument("--closure-window", type=int, default=1200,
                    help="fine steps of the torque comparison window")
    ap.add_argument("--closure-batch", type=int, default=8)
    return ap.parse_args(argv)


# ------------------------------------------------------------------ ranks
def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=300))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def aggregate(elapsed_s: float, units: float, world: int):
    """Max elapsed time and summed units over ranks (all ranks call this)."""
    if world == 1:
        return elapsed_s, units
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([elapsed_s], dtype=torch.float64, device=dev)
    u = torch.tensor([units], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(t.item()), float(u.item())


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.tmp = None

    def __enter__(self):
        self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.tmp, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.tmp.flush()
        rows = list(csv.reader(io.StringIO(open(self.tmp.name).read())))
        os.unlink(self.tmp.name)
        sm, smax, reasons = [], [], set()
        names = ["active", "hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
            except ValueError:
                continue
            for nm, v in zip(names[1:], r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        top = max(sm)
        load = [v for v in sm if v >= 0.5 * top] or sm
        return {"sm_mhz": statistics.median(load), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ CPU reference
def ref_binary():
    p = os.path.join(ROOT, "oracle", "_ref", "tcref_tc")
    return p if os.path.exists(p) else None


def cpu_reference_run(steps: int, warmup: int):
    """The reference's own integrate() on this host's cores: P concurrent
    single-rank processes on a 64x128x64 sample of the workload."""
    from simpletcsolver_b200 import ic
    nx, ny, nz = SAMPLE_GRID
    case = ic.taylor_couette(nx, ny, nz, 1.0e4)
    binary = ref_binary()
    cores = len(os.sched_getaffinity(0))
    procs = max(1, min(cores, 64))
    with tempfile.TemporaryDirectory() as td:
        d0 = ic.write_ic(case, os.path.join(td, "ic"))
        env = dict(os.environ, **ic.case_env(case))
        if binary is not None:
            kind = "reference"
            runs = [subprocess.Popen([binary, d0, str(max(1, warmup)), str(steps)], env=env, stdout=subprocess.PIPE,
                                     stderr=subprocess.DEVNULL, text=True) for _ in range(procs)]
            rates, bounds, fft, total = [], [], 0.0, 0.0
            for r in runs:
                out, _ = r.communicate(timeout=3600)
                line = [x for x in out.splitlines() if x.startswith("{")][-1]
                res = json.loads(line)
                rates.append(res["cells"] * res["steps"] / res["seconds"] / 1e6)
                # the same process with its transforms taking no time at all
                bounds.append(res["cells"] * res["steps"] / (res["seconds"] - res["fft_seconds"]) / 1e6)
                fft += res["fft_seconds"]
                total += res["seconds"]
            value = sum(rates)
            extra = {"fft_share": fft / total, "value_bound_free_fft": sum(bounds),
                     "fft_note": ("FFTW is replaced by an FP64 radix-2 shim (oracle/shim/fftw_shim.c); "
                                  "value_bound_free_fft is the throughput if the reference's transforms took no time, "
                                  "an upper bound for any FFT library")}
            sample = (f"{procs} concurrent single-rank reference processes (oracle/_ref/tcref_tc, the reference's "
                      f"own C sources), each {nx}x{ny}x{nz} at Re=1e4, {warmup} warm-up + {steps} timed steps; "
                      f"rates summed")
        else:
            kind = "port"
            from oracle import tc_numpy as tn
            prm = tn.Params(coef_dt_adv=case.coef_dt_adv, coef_dt_dif=case.coef_dt_dif)
            d = tn.load_domain(d0)
            fl = tn.load_fluid(d, d0, case.Re, case.Pr, prm)
            tn.integrate(d, fl, prm)
            t0 = time.perf_counter()
            n = max(1, min(steps, 3))
            for _ in range(n):
                tn.integrate(d, fl, prm)
            value = case.ncells * n / (time.perf_counter() - t0) / 1e6
            procs = 1
            sample = f"numpy restatement, 1 process, {nx}x{ny}x{nz}, {n} steps"
    out = {"value": value, "unit": UNIT, "cores": procs, "kind": kind, "sample": sample}
    if kind == "reference":
        out.update(extra)
    return out


def start_planar_reference(d0, case):
    """The reference's own integrate() on the planar workload's full grid,
    one single-rank process (1 warm-up + 1 timed step), in the background."""
    binary = os.path.join(ROOT, "oracle", "_ref", "tcref_planar")
    if not os.path.exists(binary):
        return None
    from simpletcsolver_b200 import ic
    env = dict(os.environ, **ic.case_env(case))
    return subprocess.Popen([binary, d0, "1", "1"], env=env, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                            text=True)


def finish_planar_reference(proc, case):
    if proc is None:
        return None
    out, _ = proc.communicate(timeout=3600)
    if proc.returncode != 0:
        return None
    res = json.loads([x for x in out.splitlines() if x.startswith("{")][-1])
    return {"value": res["cells"] * res["steps"] / res["seconds"] / 1e6, "unit": UNIT, "cores": 1,
            "kind": "reference", "fft_share": res["fft_seconds"] / res["seconds"],
            "sample": (f"oracle/_ref/tcref_planar on the full {case.nx}x{case.ny}x{case.nz} grid, one single-rank "
                       f"process, 1 warm-up + 1 timed step (the reference cannot be decomposed here)")}


# ------------------------------------------------------------------ GPU arm
def parse_grid(s):
    nx, ny, nz = (int(v) for v in s.lower().split("x"))
    return nx, ny, nz


def run_timed(lib, s, nsteps, instrument):
    """nsteps steps through tcgpu_run_timed in chunks of 64: device ms (CUDA
    events on the library's stream) and, with instrument, per-kernel ms and
    launch counts."""
    import ctypes as C
    from simpletcsolver_b200 import abi
    el = C.c_float(0.)
    kms = (C.c_double * 12)()
    kl = (C.c_int * 12)()
    dts = (C.c_double * max(nsteps, 1))()
    done = 0
    total_ms = 0.0
    ktot = [0.0] * 12
    ltot = [0] * 12
    while done < nsteps:
        n = min(64, nsteps - done)
        rc = lib.tcgpu_run_timed(C.byref(s.domain), C.byref(s.fluid), n, instrument, dts, C.byref(el), kms, kl)
        if rc != 0:
            raise RuntimeError(abi.last_error(lib))
        total_ms += el.value
        ktot = [a + b for a, b in zip(ktot, kms)]
        ltot = [a + b for a, b in zip(ltot, kl)]
        done += n
    return total_ms, ktot, ltot


def kernel_table(kms_total, kdev, klaunch, ncell, bytes_map, peak):
    per_kernel = {}
    for i, name in enumerate(KERNELS):
        if klaunch[i] == 0:
            continue
        avg = kdev[i] / klaunch[i]
        entry = {"launches": klaunch[i], "ms_total": kdev[i], "share": kdev[i] / kms_total, "ms_per_launch": avg}
        if name in bytes_map:
            entry["gbs"] = bytes_map[name] * ncell / (avg / 1e3) / 1e9
            entry["frac"] = entry["gbs"] / peak
        per_kernel[name] = entry
    return per_kernel


def gpu_config(nx, ny, nz, world):
    """The workload's config, the same for both arms."""
    return {"workload": f"taylor-couette {nx}x{ny}x{nz} Re=1e4 fp64", "grid": [nx, ny, nz], "Re": 1.0e4,
            "coef_dt_adv": 0.4, "implicit": "x", "parallelism": f"replicas{world}",
            "l2": "no flush: every field (1.09 GB at 256x1024x512) exceeds the 126 MB L2"}


def gpu_arm(args, rank, world, local):
    import ctypes as C
    from simpletcsolver_b200 import abi, build, ic
    from simpletcsolver_b200.solver import Solver
    build.build()
    lib = abi.load()
    if lib.tcgpu_set_device(local) != 0:
        raise RuntimeError(abi.last_error(lib))
    lib.tcgpu_run_timed.argtypes = [C.POINTER(abi.DomainT), C.POINTER(abi.FluidT), C.c_int, C.c_int,
                                    abi.c_double_p, C.POINTER(C.c_float), C.c_double * 12, C.c_int * 12]
    nx, ny, nz = parse_grid(args.grid)
    case = ic.taylor_couette(nx, ny, nz, 1.0e4)
    td = tempfile.mkdtemp(prefix="tcbench")
    d0 = os.path.join(td, "ic")
    # the seeded initial field generated on the device (no 1.1 GB NPY per field)
    s = Solver.from_case(case, d0, lib=lib)
    s.set_coherence(abi.PIN_HOST)
    s.push()
    K, W = args.steps, args.warmup
    s.run(W)                                     # warm-up, graph capture
    ncell = case.ncells

    import torch
    barrier(world)
    if torch.cuda.is_available():
        torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        ms, _, launches = run_timed(lib, s, K, 0)
    barrier(world)
    if torch.cuda.is_available():
        torch.cuda.synchronize()
    elapsed, units = aggregate(ms / 1e3, ncell * K, world)
    value = units / elapsed / 1e6

    # per-kernel accounting: events around every launch of K instrumented steps
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peaks = json.load(open(peaks_path)) if os.path.exists(peaks_path) else {}
    peak = float(peaks.get("hbm_gbs", 6650.0))
    kms_total, kdev, klaunch = run_timed(lib, s, K, 1)
    per_kernel = kernel_table(kms_total, kdev, klaunch, ncell, BYTES_PER_CELL, peak)
    dom = max((k for k in per_kernel if k in BYTES_PER_CELL), key=lambda k: per_kernel[k]["ms_total"])
    achieved = per_kernel[dom]["gbs"]
    traffic = measured_traffic(dom, ncell)
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic,
                "algorithmic_bytes_per_launch": BYTES_PER_CELL[dom] * ncell,
                "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"}
    step_model = MODEL_BYTES_PER_CELL_STEP * ncell / (ms / K / 1e3) / 1e9

    e2e = None
    if not args.no_e2e:
        t0 = time.perf_counter()
        for _ in range(K):
            s.integrate()
        el = time.perf_counter() - t0
        e_el, e_units = aggregate(el, ncell * K, world)
        nf = (nx + 1) * (ny + 2) * (nz + 2)
        nc = (nx + 2) * (ny + 2) * (nz + 2)
        e2e = {"value": e_units / e_el / 1e6, "unit": UNIT, "h2d_bytes_per_step": (nf + 4 * nc) * 8,
               "d2h_bytes_per_step": (nf + 5 * nc) * 8, "timing": "host wall clock around synchronous integrate()"}
        # the resident API end to end: the state stays on the device for K steps
        # (tcgpu_run), then every field comes back once, as before a save
        s.set_coherence(abi.NO_COHERENCE | abi.PIN_HOST)
        s.push()
        t0 = time.perf_counter()
        s.run(K)
        s.pull(abi.FIELDS)
        el = time.perf_counter() - t0
        r_el, r_units = aggregate(el, ncell * K, world)
        e2e["resident_api"] = {"value": r_units / r_el / 1e6, "unit": UNIT, "steps": K,
                               "d2h_bytes": (nf + 5 * nc) * 8,
                               "timing": "host wall clock around tcgpu_run(K steps) + one tcgpu_pull of all fields"}
    s.release()
    gpu_launches = sum(launches)

    fp32 = None
    if not args.no_fp32:
        fp32 = fp32_storage_arm(args, lib, d0, case, world, peak, value)
        fp32["gpu_launches"] = fp32.pop("_launches")

    planar = None
    if not args.no_planar:
        planar = planar_arm(args, lib, world, peak)

    clo = None
    if not args.no_closure and nx % 32 == 0 and ny % 64 == 0 and nz % 4 == 0:
        clo = closure_arm(args, lib, d0, case, peaks)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference_run(max(2, min(args.steps, 5)), 1)
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": elapsed * 1e3 / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic: seeded noisy circular-Couette field generated on the device (no dataset involved)",
            "config": gpu_config(nx, ny, nz, world),
            "roofline": roofline,
            "step_model": {"bytes_per_cell_step": MODEL_BYTES_PER_CELL_STEP, "achieved_gbs": step_model,
                           "frac": step_model / peak},
            "kernels": per_kernel,
            "fp32_storage": fp32,
            "closure": clo,
            "planar": planar,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "clocks": clk.summary(),
            "gpu_launches": gpu_launches,
        }
        print(json.dumps(out))
    return 0


def fp32_storage_arm(args, lib, d0, case, world, peak, value64):
    """The FP32-storage form on the same workload: throughput (same timing as
    the FP64 arm) and, over --accuracy-steps steps from the same initial field,
    its error against the FP64 path: relative L2 of every field, max
    divergence, inner-wall torque (the momentum energy injection; the outer
    wall is at rest) and Nusselt number (torque / its laminar value)."""
    from simpletcsolver_b200 import abi
    from simpletcsolver_b200.solver import Solver
    K, W = args.steps, args.warmup
    ncell = case.ncells
    s = Solver.from_case(case, d0, lib=lib, storage=4)
    s.push()
    s.run(W)
    ms, _, launches = run_timed(lib, s, K, 0)
    elapsed, units = aggregate(ms / 1e3, ncell * K, world)
    value = units / elapsed / 1e6
    kms_total, kdev, klaunch = run_timed(lib, s, K, 1)
    per_kernel = kernel_table(kms_total, kdev, klaunch, ncell, BYTES_PER_CELL_FP32, peak)
    s.release()
    step_model = MODEL_BYTES_PER_CELL_STEP_FP32 * ncell / (ms / K / 1e3) / 1e9
    out = {"value": value, "unit": UNIT, "ms_per_step": elapsed * 1e3 / K, "steps": K,
           "dtype": "f32 storage (ux, uy, uz, t, sources, spectra); p, psi and arithmetic f64",
           "speedup_vs_fp64": value / value64,
           "step_model": {"bytes_per_cell_step": MODEL_BYTES_PER_CELL_STEP_FP32, "achieved_gbs": step_model,
                          "frac": step_model / peak},
           "kernels": per_kernel, "_launches": sum(launches)}
    n = args.accuracy_steps
    if n > 0:
        runs = {}
        for storage in (8, 4):
            s = Solver.from_case(case, d0, lib=lib, storage=storage)
            try:
                s.push()
                dts = s.run(n)
                s.pull(abi.FIELDS)
                runs[storage] = {f: s.field(f)[1:-1, 1:-1].copy() for f in ("ux", "uy", "uz", "t", "p")}
                runs[storage]["diag"] = s.diagnostics()
                runs[storage]["time"] = float(np.sum(dts))
            finally:
                s.release()
        a, b = runs[8], runs[4]
        l2 = {}
        for f in ("ux", "uy", "uz", "t", "p"):
            x, y = b[f], a[f]
            if f == "p":
                x, y = x - x.mean(), y - y.mean()
            l2[f] = float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))
        tq64, tq32 = a["diag"]["injection_u"], b["diag"]["injection_u"]
        lam = laminar_injection(case)
        out["accuracy"] = {
            "steps": n, "rel_l2": l2,
            "divmax": {"fp64": a["diag"]["divmax"], "fp32_storage": b["diag"]["divmax"]},
            "torque": {"fp64": tq64, "fp32_storage": tq32, "rel_err": abs(tq32 - tq64) / abs(tq64)},
            "nusselt": {"fp64": tq64 / lam, "fp32_storage": tq32 / lam,
                        "rel_err": abs(tq32 - tq64) / abs(tq64)},
            "sim_time": {"fp64": a["time"], "fp32_storage": b["time"]},
        }
    return out


MODEL_BYTES_PER_CELL_STEP_PLANAR = 1512   # + y and z implicit solves and the increment round trip per substep


def planar_arm(args, lib, world, peak):
    """The planar channel workload (192x512x256, Re = 2000, Pr = 1, walls at
    -0.5 / +0.5, scalar 1 / 0, implicit diffusion in x, y and z): device time
    of K steps in FP64 and in the FP32-storage form, timed like the main arm."""
    from simpletcsolver_b200 import abi, ic
    from simpletcsolver_b200.solver import Solver
    case = ic.PLANAR
    d0 = ic.write_ic(case, os.path.join(tempfile.mkdtemp(prefix="tcplanar"), "ic"))
    K, W = args.steps, args.warmup
    out = {"workload": f"planar channel {case.nx}x{case.ny}x{case.nz} Re=2000 Pr=1 implicit xyz",
           "steps": K, "bytes_per_cell_step_model": MODEL_BYTES_PER_CELL_STEP_PLANAR}
    ref = start_planar_reference(d0, case) if (world == 1 and not args.no_cpu_baseline) else None
    for storage, key in ((8, "fp64"), (4, "fp32_storage")):
        s = Solver.from_ic(d0, case=case, lib=lib, storage=storage)
        try:
            s.set_coherence(abi.NO_COHERENCE)
            s.push()
            s.run(W)
            ms, _, _ = run_timed(lib, s, K, 0)
            elapsed, units = aggregate(ms / 1e3, case.ncells * K, world)
            out[key] = {"value": units / elapsed / 1e6, "unit": UNIT, "ms_per_step": elapsed * 1e3 / K,
                        "divmax": s.diagnostics()["divmax"]}
            if storage == 8:
                out[key]["step_model_frac"] = (MODEL_BYTES_PER_CELL_STEP_PLANAR * case.ncells / (ms / K / 1e3)
                                               / 1e9 / peak)
        finally:
            s.release()
    cpu = finish_planar_reference(ref, case)
    if cpu is not None:
        # the same grid and configuration on both arms: one core of the reference against one GPU
        out["cpu_reference_same_grid"] = cpu
        out["fp64"]["vs_cpu_reference_1core"] = out["fp64"]["value"] / cpu["value"]
    return out


CLOSURE_FLOP_PER_CELL = 2 * 27 * (4 * 32 + 32 * 32 + 32 * 32 + 32 * 3)   # one forward, real channels


def closure_arm(args, lib, d0, case, peaks):
    """Learned closure on the 4x-coarsened grid: pairs from the fine FP64 run,
    training on 3/4 of them (every 4th held out), the network's forward pass
    timed against the tensor-core peak, and a torque comparison over a window
    of --closure-window fine steps: the fine run, the coarse run with the
    closure and without it, all started from the same (restricted) state."""
    import torch
    from simpletcsolver_b200 import abi, closure
    from simpletcsolver_b200.solver import Solver
    td = os.path.dirname(d0)
    dc = closure.write_coarse_ic(case, os.path.join(td, "coarse"))
    cc = closure.coarse_case(case)
    fine = Solver.from_case(case, d0, lib=lib)
    ca = Solver.from_ic(dc, case=cc, lib=lib)
    cb = Solver.from_ic(dc, case=cc, lib=lib)
    cf = Solver.from_ic(dc, case=cc, lib=lib)     # the fine run restricted, for the coarse-grid diagnostics
    cd = Solver.from_ic(dc, case=cc, lib=lib)     # closure forcing recomputed every RK substep
    out = {"grid_fine": [case.nx, case.ny, case.nz], "grid_coarse": [cc.nx, cc.ny, cc.nz]}
    try:
        for s in (fine, ca, cb, cf, cd):
            closure.resident(s)
        fine.run(args.closure_warm)
        in_scale = (0.05, 1.0, 0.05)
        t0 = time.perf_counter()
        data, t_scale = closure.generate(fine, ca, cb, args.closure_pairs, 8, in_scale=in_scale)
        gen_s = time.perf_counter() - t0
        n = data.n
        train = [q for q in range(n) if q % 4]
        held = [q for q in range(n) if q % 4 == 0]
        net = closure.ClosureNet(lib, (cc.nx, cc.ny, cc.nz), seed=0)
        before = closure.relative_error(net, data, held)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        batch = args.closure_batch
        hist = closure.train(net, data, train, epochs=args.closure_epochs, batch=batch, lr=2e-3)
        # the learned wall model (near-wall reconstruction for the torque), fitted
        # on the same training pairs; its injection formula checked against the
        # fine solver's own on the fine field
        wm = closure.WallModel.fit(data, train, fine, ca)
        fine_formula = closure.WallModel.fine_injection(wm, fine.radial_slab("uy", 1, 1))
        fine_diag = fine.diagnostics()["injection_u"]
        held_err = []
        for q in held:
            pred = wm.predict(data.wall_x[q])
            tgt = closure.block_mean(data.wall_y[q], ca).ravel()
            held_err.append(float(np.sqrt(np.mean((pred - tgt) ** 2)) / np.sqrt(np.mean(tgt ** 2))))
        train_s = time.perf_counter() - t0
        err_train = closure.relative_error(net, data, train)
        err_held = closure.relative_error(net, data, held)
        # forward pass on the tensor cores: CUDA events on the stream it runs on;
        # the median of 7 repeats of 20 passes, SM clocks sampled meanwhile
        # (the passes follow the training run, so the clock it left matters)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        x = data.X[0]
        for _ in range(3):
            net.forward(x, keep=False)
        fwd_reps = []
        with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as fclk:
            for _ in range(7):
                e0.record()
                for _ in range(20):
                    net.forward(x, keep=False)
                e1.record()
                torch.cuda.synchronize()
                fwd_reps.append(e0.elapsed_time(e1) / 20)
        fwd_ms = statistics.median(fwd_reps)
        tflops = CLOSURE_FLOP_PER_CELL * net.ncell / (fwd_ms / 1e3) / 1e12
        peak = float(peaks.get("bf16_tflops", 1590.0))
        # torque window: fine, coarse with and without the closure from one state
        for s in (ca, cb, cd):
            s._check(lib.tcgpu_coarsen(C.byref(fine.domain), C.byref(fine.fluid), C.byref(s.domain),
                                       C.byref(s.fluid)), "coarsen")
        def restricted_torque():
            cf._check(lib.tcgpu_coarsen(C.byref(fine.domain), C.byref(fine.fluid), C.byref(cf.domain),
                                        C.byref(cf.fluid)), "coarsen")
            return cf.diagnostics()["injection_u"], wm.torque(cf)

        r0 = restricted_torque()
        ft, fq, rq, rw = [0.0], [fine.diagnostics()["injection_u"]], [r0[0]], [r0[1]]
        fine_s = 0.0
        for _ in range(max(1, args.closure_window // 10)):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ft.append(ft[-1] + float(np.sum(fine.run(10))))
            fine_s += time.perf_counter() - t0
            fq.append(fine.diagnostics()["injection_u"])
            r = restricted_torque()
            rq.append(r[0])
            rw.append(r[1])
        # the coarse runs from the window's start state: closure forcing per step
        # (timed, its per-step diagnostics included), no closure, forcing per RK substep
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        at, aq, aw = closure.run_coarse(ca, ft[-1], net, in_scale, t_scale, wall_model=wm)
        torch.cuda.synchronize()
        coarse_s = time.perf_counter() - t0
        bt, bq, bw = closure.run_coarse(cb, ft[-1], wall_model=wm)
        dtm, dq, dw = closure.run_coarse(cd, ft[-1], net, in_scale, t_scale, wall_model=wm, per_substep=True)
        tq_f = closure.time_average(ft, fq)
        tq_r = closure.time_average(ft, rq)
        tq_c = closure.time_average(at, aq)
        tq_p = closure.time_average(bt, bq)
        tw_r = closure.time_average(ft, rw)
        tw_c = closure.time_average(at, aw)
        tw_p = closure.time_average(bt, bw)
        tw_d = closure.time_average(dtm, dw)
        # mean azimuthal velocity profile at the end of the window (coarse grid)
        prof = {}
        for name, s in (("restricted_fine", cf), ("closure", ca), ("plain", cb), ("closure_per_substep", cd)):
            s.pull(abi.UY)
            prof[name] = s.field("uy")[1:-1, 1:-1, 1:-1].mean(axis=(0, 1))
        perr = lambda a: float(np.linalg.norm(a - prof["restricted_fine"]) / np.linalg.norm(prof["restricted_fine"]))
        out.update({
            "pairs": n, "pair_gap_fine_steps": 8, "generate_s": gen_s,
            "training": {"epochs": args.closure_epochs, "samples": len(train), "batch": batch, "seconds": train_s,
                         "loss_first": hist[0], "loss_last": hist[-1]},
            "apriori_rel_error": {"no_closure": 1.0, "train": err_train, "held_out": err_held,
                                  "held_out_untrained": before},
            "forward": {"ms": fwd_ms, "repeats_ms": fwd_reps, "clocks": fclk.summary(), "tflops": tflops,
                        "peak_tflops": peak, "frac": tflops / peak,
                        "flop_per_cell": CLOSURE_FLOP_PER_CELL,
                        "peak_source": "measured" if "bf16_tflops" in peaks else "fallback"},
            "wall_model": {"weights": [float(v) for v in wm.w], "fit_samples": wm.samples,
                           "fit_rms": wm.fit_rms, "held_out_rel_rms": float(np.mean(held_err)),
                           "formula_vs_fine_injection": abs(fine_formula - fine_diag) / abs(fine_diag)},
            "torque_window": {
                "sim_time": ft[-1], "fine_steps": 10 * (len(ft) - 1), "coarse_steps": len(at) - 1,
                "fine": tq_f,
                # the coarse grid's torque with the learned wall model (the closure's estimator)
                "restricted_fine": tw_r, "coarse_closure": tw_c, "coarse_plain": tw_p,
                "coarse_closure_per_substep": tw_d,
                "rel_err_closure": abs(tw_c - tq_f) / abs(tq_f), "rel_err_plain": abs(tw_p - tq_f) / abs(tq_f),
                "rel_err_closure_per_substep": abs(tw_d - tq_f) / abs(tq_f),
                "rel_err_restricted_fine": abs(tw_r - tq_f) / abs(tq_f),
                # the reference's injection formula applied on the coarse grid as it is
                "raw_estimator": {
                    "restricted_fine": tq_r, "coarse_closure": tq_c, "coarse_plain": tq_p,
                    "rel_err_closure": abs(tq_c - tq_f) / abs(tq_f), "rel_err_plain": abs(tq_p - tq_f) / abs(tq_f),
                    "rel_err_closure_vs_restricted": abs(tq_c - tq_r) / abs(tq_r),
                    "rel_err_plain_vs_restricted": abs(tq_p - tq_r) / abs(tq_r)},
                "mean_uy_profile_rel_err": {"closure": perr(prof["closure"]), "plain": perr(prof["plain"]),
                                            "closure_per_substep": perr(prof["closure_per_substep"])},
                "wall_s_fine": fine_s, "wall_s_coarse_closure": coarse_s,
                "speedup_vs_fine": (fine_s / ft[-1]) / (coarse_s / max(at[-1], 1e-30)),
            },
        })
    finally:
        for s in (fine, ca, cb, cf, cd):
            s.release()
    return out


def laminar_injection(case):
    """Energy injection of circular Couette flow in the same box:
    2/Re ri^2 ro^2 / (ro^2 - ri^2) (ui/ri)^2 ly lz, the normalisation of the
    reference's Nusselt number (balance_main.py:14-21); ri = 1, ui = uy_xm."""
    ri, ro = 1.0, 1.0 + case.lx
    return (2.0 / case.Re * ri ** 2 * ro ** 2 / (ro ** 2 - ri ** 2) * (case.uy_xm / ri) ** 2
            * case.ly * case.lz)


def measured_traffic(kernel: str, ncell: int):
    """DRAM bytes per launch from the committed ncu summary of that kernel
    (profiles/*.txt lines 'kernel: NAME dram_bytes_per_cell: X')."""
    pdir = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pdir):
        return None
    for fn in sorted(os.listdir(pdir)):
        if not fn.endswith(".txt"):
            continue
        for line in open(os.path.join(pdir, fn)):
            parts = line.split()
            if len(parts) >= 4 and parts[0] == "kernel:" and parts[1] == kernel and parts[2] == "dram_bytes_per_cell:":
                return float(parts[3]) * ncell
    return None


def reference_arm(args, rank, world):
    if rank != 0:
        return 0
    cpu = cpu_reference_run(args.steps, args.warmup)
    nx, ny, nz = parse_grid(args.grid)
    # milliseconds per step of the whole workload at the measured throughput
    ms_per_step = nx * ny * nz / (cpu["value"] * 1e6) * 1e3
    out = {"impl": "reference", "metric": METRIC, "value": cpu["value"], "unit": UNIT, "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic: seeded noisy circular-Couette field",
           "config": gpu_config(nx, ny, nz, world),
           "sample": {"grid": list(SAMPLE_GRID), "note": cpu["sample"]},
           "cpu_baseline": cpu,
           "e2e": {"value": cpu["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


def main(argv=None):
    args = parse_args(argv)
    rank, world, local = dist_setup()
    try:
        if args.impl == "reference":
            return reference_arm(args, rank, world)
        return gpu_arm(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
