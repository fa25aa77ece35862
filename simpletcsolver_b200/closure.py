"""Learned closure of a 4x-coarsened Taylor-Couette solver (no counterpart in
the reference).

A 3D convolutional network (four 3x3x3 layers, 4 -> 32 -> 32 -> 32 -> 3
channels, GELU, zero padding at the walls, periodic in y and z) maps the
coarse state (ux averaged to the centre, uy, uz, a radial coordinate) to a
forcing of ux, uy, uz that the coarse solver adds to its explicit terms in
every predict, held over one step. It is trained on pairs made by the
fine-grid solver itself: the fine state restricted to the coarse grid at t,
and the gap after tau between the restricted fine state and one coarse step
from it, (restrict(u_fine(t + tau)) - coarse_step(restrict(u_fine(t)), tau)) / tau.

Every arithmetic operation runs in libtcgpu: the convolutions and their
gradients on the tensor cores (BF16 weights and activations, FP32
accumulation), the loss, Adam, the restriction and the forcing hand-off.
torch only allocates device memory.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import abi

# (real input channels, padded, real output channels, padded)
LAYERS = ((4, 16, 32, 32), (32, 32, 32, 32), (32, 32, 32, 32), (32, 32, 3, 16))
NIN = 16      # channels of the network input buffer
NOUT = 3


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("the closure network needs a CUDA device")
    return torch


def _p(t, offset_elems: int = 0) -> C.c_void_p:
    return C.c_void_p(t.data_ptr() + offset_elems * t.element_size())


class ClosureNet:
    """Parameters (FP32 master copy, flat: W1, b1, ..., W4, b4 with
    W[t][co][ci], t = 9 (dz+1) + 3 (dy+1) + (dx+1)), their BF16 images,
    activations for one sample of a grid (nx, ny, nz), gradients and Adam
    moments."""

    def __init__(self, lib, grid, seed: int = 0, last_scale: float = 0.1):
        torch = _torch()
        self.lib = lib
        self.nx, self.ny, self.nz = grid
        if self.nx % 8 or self.ny % 16:
            raise ValueError("closure grid: nx must be a multiple of 8 and ny of 16")
        self.ncell = self.nx * self.ny * self.nz
        rng = np.random.default_rng(seed)
        chunks, self.woff, self.boff = [], [], []
        off = 0
        for li, (cin, _, cout, _) in enumerate(LAYERS):
            std = math.sqrt(2.0 / (27 * cin)) * (last_scale if li == len(LAYERS) - 1 else 1.0)
            w = rng.normal(0.0, std, size=(27, cout, cin)).astype(np.float32)
            self.woff.append(off)
            off += w.size
            self.boff.append(off)
            off += cout
            chunks += [w.ravel(), np.zeros(cout, np.float32)]
        self.nparam = off
        dev = "cuda"
        self.params = torch.tensor(np.concatenate(chunks), device=dev)
        self.grads = torch.zeros_like(self.params)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        bf = torch.bfloat16
        self.wf = [torch.zeros(27 * cp * op, dtype=bf, device=dev) for (_, cp, _, op) in LAYERS]
        self.wb = [torch.zeros(27 * cp * op, dtype=bf, device=dev) for (_, cp, _, op) in LAYERS]
        n = self.ncell
        self.a = [torch.zeros(n * NIN, dtype=bf, device=dev)] + [torch.zeros(n * 32, dtype=bf, device=dev)
                                                                  for _ in range(3)]
        self.z = [None] + [torch.zeros(n * 32, dtype=bf, device=dev) for _ in range(3)]
        self.g = [None] + [torch.zeros(n * 32, dtype=bf, device=dev) for _ in range(3)] + \
                 [torch.zeros(n * 16, dtype=bf, device=dev)]
        self.out = torch.zeros(n * NOUT, dtype=torch.float32, device=dev)
        ws = max(lib.tcgpu_nn_wgrad_workspace(self.nx, self.ny, self.nz, op) for (_, _, _, op) in LAYERS)
        self.ws = torch.zeros(ws // 4 + 4, dtype=torch.float32, device=dev)
        self.ws_bytes = ws
        self.loss = torch.zeros(1, dtype=torch.float64, device=dev)
        self.adam_steps = 0
        self.pack()

    # ------------------------------------------------------------ plumbing
    def _ck(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what}: {self.lib.tcgpu_nn_last_error().decode()}")

    def state_dict(self) -> dict:
        return {"params": self.params.detach().cpu().numpy().copy(), "adam_steps": self.adam_steps}

    def load_state(self, params: np.ndarray, stream=None):
        torch = _torch()
        self.params.copy_(torch.from_numpy(np.asarray(params, np.float32)))
        self.pack(stream)

    def pack(self, stream=None):
        for li, (cin, cp, cout, op) in enumerate(LAYERS):
            self._ck(self.lib.tcgpu_nn_pack_weights(_p(self.params, self.woff[li]), cin, cout, cp, op,
                                                     _p(self.wf[li]), _p(self.wb[li]), stream), "pack_weights")

    # ------------------------------------------------------------ passes
    def forward(self, x=None, stream=None, keep: bool = True):
        """Network output (FP32 [cell][3] in self.out) of input x (BF16
        [cell][16]; default self.a[0]); keep: store the pre-activations the
        backward pass needs."""
        lib = self.lib
        src = x if x is not None else self.a[0]
        for li in range(3):
            cin, cp, cout, op = LAYERS[li]
            self._ck(lib.tcgpu_nn_conv3(0, cp, op, self.nx, self.ny, self.nz, _p(src), _p(self.wf[li]),
                                        _p(self.params, self.boff[li]), None, _p(self.a[li + 1]),
                                        _p(self.z[li + 1]) if keep else None, None, 0, stream), "conv3 forward")
            src = self.a[li + 1]
        cin, cp, cout, op = LAYERS[3]
        self._ck(lib.tcgpu_nn_conv3(1, cp, op, self.nx, self.ny, self.nz, _p(src), _p(self.wf[3]),
                                    _p(self.params, self.boff[3]), None, None, None, _p(self.out), NOUT, stream),
                 "conv3 forward (output layer)")
        return self.out

    def backward(self, target, x=None, stream=None, accumulate: bool = False, weight=None):
        """Gradients of the MSE of self.out against target (FP32 [cell][3]) into
        self.grads (accumulate: add to them); adds the loss to self.loss."""
        lib = self.lib
        beta = 1.0 if accumulate else 0.0
        self._ck(lib.tcgpu_nn_mse(_p(self.out), _p(target), _p(weight) if weight is not None else None,
                                  self.ncell, NOUT, 16, _p(self.g[4]), _p(self.loss), stream), "mse")
        inputs = [x if x is not None else self.a[0], self.a[1], self.a[2], self.a[3]]
        for li in (3, 2, 1, 0):
            cin, cp, cout, op = LAYERS[li]
            self._ck(lib.tcgpu_nn_conv3_wgrad(cp, op, cin, cout, self.nx, self.ny, self.nz, _p(inputs[li]),
                                              _p(self.g[li + 1]), _p(self.grads, self.woff[li]),
                                              _p(self.grads, self.boff[li]), beta, _p(self.ws), self.ws_bytes,
                                              stream), "conv3 weight gradient")
            if li > 0:
                self._ck(lib.tcgpu_nn_conv3(2, op, cp, self.nx, self.ny, self.nz, _p(self.g[li + 1]),
                                            _p(self.wb[li]), None, _p(self.z[li]), _p(self.g[li]), None, None, 0,
                                            stream), "conv3 input gradient")

    def adam(self, lr: float = 1e-3, stream=None):
        self.adam_steps += 1
        self._ck(self.lib.tcgpu_nn_adam(_p(self.params), _p(self.grads), _p(self.m), _p(self.v), self.nparam, lr,
                                        0.9, 0.999, 1e-8, self.adam_steps, stream), "adam")
        self.pack(stream)


# ---------------------------------------------------------------- coarse grid
def coarse_case(case, factor: int = 4):
    """The case on the grid coarser by factor in every direction."""
    from dataclasses import replace
    if case.nx % factor or case.ny % factor or case.nz % factor:
        raise ValueError("grid not divisible by the coarsening factor")
    return replace(case, nx=case.nx // factor, ny=case.ny // factor, nz=case.nz // factor)


def write_coarse_ic(case, dest: str) -> str:
    """Initial-condition directory of the 4x-coarser grid (its radial faces
    are every 4th fine face; the fields are overwritten by tcgpu_coarsen)."""
    from . import ic
    cc = coarse_case(case)
    xf_f, _ = ic.radial_grid(case)
    xf_c, _ = ic.radial_grid(cc)
    if np.max(np.abs(xf_c - xf_f[::4])) > 1e-14:
        raise ValueError("the coarse radial faces are not every 4th fine face")
    return ic.write_ic(cc, dest)


def resident(s) -> None:
    """Device-resident state: push once, no host copies from then on."""
    s.set_coherence(abi.NO_COHERENCE)
    s.push()


def stream_of(s) -> C.c_void_p:
    return C.c_void_p(s.lib.tcgpu_stream(C.byref(s.domain), C.byref(s.fluid)))


def coarse_step(s, dt: float) -> None:
    """One RK3 step of prescribed size dt through the reference's stage entry
    points (src/integrate.c:15-32)."""
    for rk in range(3):
        s.predict(rk, dt)
        s.compute_potential(rk, dt)
        s.correct_velocity(rk, dt)
        s.update_pressure(rk, dt)


def _d3(v) -> "C.Array":
    return (C.c_double * 3)(*[float(x) for x in v])


class Dataset:
    """Closure training pairs on the device: inputs X[s] (BF16 [cell][16]) and
    normalised targets T[s] (FP32 [cell][3], divided by t_scale), with the
    time gap tau of each pair."""

    def __init__(self, ncell: int, nmax: int):
        torch = _torch()
        self.X = torch.zeros(nmax, ncell * NIN, dtype=torch.bfloat16, device="cuda")
        self.T = torch.zeros(nmax, ncell * NOUT, dtype=torch.float32, device="cuda")
        self.tau = []
        self.n = 0
        # wall-model pairs: the restricted state's first WALL_DEPTH radial cells
        # of uy at the inner wall, and the fine state's first-cell uy there
        self.wall_x = []
        self.wall_y = []


def generate(fine, coarse_a, coarse_b, nsamples: int, gap: int, in_scale, data: Dataset | None = None,
             t_scale=None, max_sub: int = 8):
    """Pairs from the fine run: every `gap` fine steps, restrict the fine state
    into coarse_a (input), advance the fine solver by n steps (n fine time
    steps fit in one coarse time step, n <= max_sub), step coarse_a once with
    their total tau, restrict the new fine state into coarse_b and take the
    target (b - a) / tau. All three solvers are device-resident. The targets
    are divided by t_scale (per channel; default: their rms over all pairs)."""
    lib = fine.lib
    torch = _torch()
    ncell = coarse_a.nx * coarse_a.ny * coarse_a.nz
    data = data or Dataset(ncell, nsamples)
    one = torch.zeros(ncell * NOUT, dtype=torch.float32, device="cuda")
    raw = []
    for _ in range(nsamples):
        if gap > 0:
            fine.run(gap)
        coarse_a._check(lib.tcgpu_coarsen(C.byref(fine.domain), C.byref(fine.fluid), C.byref(coarse_a.domain),
                                          C.byref(coarse_a.fluid)), "coarsen")
        x = data.X[data.n + len(raw)]
        coarse_a._check(lib.tcgpu_closure_input(C.byref(coarse_a.domain), C.byref(coarse_a.fluid),
                                                _d3(in_scale), NIN, _p(x)), "closure_input")
        data.wall_x.append(coarse_a.radial_slab("uy", 1, WALL_DEPTH))
        data.wall_y.append(fine.radial_slab("uy", 1, 1)[:, :, 0])
        dt_c = coarse_a.decide_dt()
        dt_f = fine.decide_dt()
        n = int(max(1, min(max_sub, math.floor(dt_c / dt_f))))
        tau = float(np.sum(fine.run(n)))
        coarse_step(coarse_a, tau)
        coarse_b._check(lib.tcgpu_coarsen(C.byref(fine.domain), C.byref(fine.fluid), C.byref(coarse_b.domain),
                                          C.byref(coarse_b.fluid)), "coarsen")
        coarse_a._check(lib.tcgpu_closure_target(C.byref(coarse_a.domain), C.byref(coarse_a.fluid),
                                                 C.byref(coarse_b.fluid), tau, _p(one)), "closure_target")
        raw.append(one.cpu().numpy().reshape(-1, NOUT).copy())
        data.tau.append(tau)
    if t_scale is None:
        ss = sum(np.sum(r.astype(np.float64) ** 2, axis=0) for r in raw)
        t_scale = np.sqrt(ss / (len(raw) * ncell)) + 1e-30
    for r in raw:
        data.T[data.n].copy_(torch.from_numpy((r / np.asarray(t_scale, np.float32)[None, :]).ravel()))
        data.n += 1
    return data, np.asarray(t_scale, dtype=np.float64)


# ---------------------------------------------------------------- wall model
WALL_DEPTH = 3   # coarse radial cells the wall model reads


class WallModel:
    """Learned near-wall reconstruction for the coarse grid's torque.

    The energy injection at the inner wall (src/logging/injection.c:55-73) is,
    per wall face, affine in the first cell's uy: with ux = 0 on the wall face
    lyx0 vanishes, lyx1 = c1 uy(1) (lyx.c:70-83, the wall weight of uy(0) is 0)
    and lxy = (uy(1) - uy(0)) / hx (lxy.c:19-49), so
        face = nu (-J / hx) uy(0) [(c1 + 1 / hx) uy(1) - uy(0) / hx]
    with J = JDXF(1), hx = HXXF(1) of the grid it is evaluated on. A coarse
    face covers 4 x 4 fine faces; the coarse grid's own first-cell value
    (a mean over 4 fine cells in x) misses the wall gradient the fine cells
    resolve. The model predicts the mean fine first-cell uy over the 16 fine
    faces of each coarse face from the coarse uy(1..WALL_DEPTH) there, linear
    with an intercept, fitted by least squares on the training pairs (coarse
    state = the restricted fine state, target = the fine state at the same
    time). The torque of a coarse state is then the fine-grid injection of the
    predicted first-cell values. The outer wall is at rest (uy(nx+1) = 0), so
    its term is zero."""

    def __init__(self, fine, coarse, weights):
        self.w = np.asarray(weights, dtype=np.float64)
        d = fine.domain
        self.nu = 1.0 / fine.fluid.Re
        J, hx = d.jdxf[0], d.hxxf[0]   # JDXF(1), HXXF(1): face arrays start at face 1 (array_macros/domain)
        c1 = -0.5 / J * (-d.jdxc[0] / d.hxxc[0] + d.jdxc[1] / d.hxxc[1])
        self.uw = fine_wall_velocity(fine)
        k = self.nu * (-J / hx) * self.uw
        self.a = k * (-self.uw / hx)         # per fine face: a + b uy(1)
        self.b = k * (c1 + 1.0 / hx)
        self.ratio = (fine.ny // coarse.ny) * (fine.nz // coarse.nz)

    @staticmethod
    def fine_injection(model, uy1) -> float:
        return float(model.a * uy1.size + model.b * np.sum(uy1))

    @classmethod
    def fit(cls, data: "Dataset", idx, fine, coarse):
        X = np.concatenate([data.wall_x[s].reshape(-1, WALL_DEPTH) for s in idx])
        y = np.concatenate([block_mean(data.wall_y[s], coarse).ravel() for s in idx])
        A = np.hstack([X, np.ones((X.shape[0], 1))])
        w, *_ = np.linalg.lstsq(A, y, rcond=None)
        m = cls(fine, coarse, w)
        m.fit_rms = float(np.sqrt(np.mean((A @ w - y) ** 2)))
        m.samples = int(X.shape[0])
        return m

    def predict(self, feats) -> np.ndarray:
        return feats.reshape(-1, WALL_DEPTH) @ self.w[:WALL_DEPTH] + self.w[WALL_DEPTH]

    def torque(self, s) -> float:
        """Inner-wall energy injection of the coarse state s with the predicted
        fine first-cell values."""
        pred = self.predict(s.radial_slab("uy", 1, WALL_DEPTH))
        return float(self.ratio * (self.a * pred.size + self.b * np.sum(pred)))


def fine_wall_velocity(s) -> float:
    """uy on the inner wall (the solver's wall value, read from the device)."""
    return float(s.radial_slab("uy", 0, 1)[0, 0, 0])


def block_mean(a, coarse):
    """Mean over the fine (k, j) blocks of each coarse wall face."""
    nz, ny = a.shape
    fz, fy = nz // coarse.nz, ny // coarse.ny
    return a.reshape(coarse.nz, fz, coarse.ny, fy).mean(axis=(1, 3))


def train(net: ClosureNet, data: Dataset, idx, epochs: int, batch: int = 8, lr: float = 1e-3, seed: int = 0,
          log=None, lr_final: float | None = None):
    """Adam over the samples idx (a batch accumulates its samples'
    gradients), the learning rate decaying from lr to lr_final (default
    lr / 10) along a half cosine over the epochs, so that the last epochs take
    small steps; returns the mean loss of each epoch."""
    torch = _torch()
    rng = np.random.default_rng(seed)
    lo = lr / 10 if lr_final is None else lr_final
    hist = []
    for ep in range(epochs):
        order = rng.permutation(np.asarray(idx))
        net.loss.zero_()
        lr_ep = lo + (lr - lo) * 0.5 * (1.0 + math.cos(math.pi * ep / max(epochs, 1)))
        for b0 in range(0, len(order), batch):
            chunk = order[b0:b0 + batch]
            for q, s in enumerate(chunk):
                net.forward(data.X[s])
                net.backward(data.T[s], x=data.X[s], accumulate=q > 0)
            net.adam(lr_ep)
        torch.cuda.synchronize()
        hist.append(net.loss.item() / len(order))
        if log:
            log(ep, hist[-1])
    return hist


def relative_error(net: ClosureNet, data: Dataset, idx) -> float:
    """sum |f - t|^2 / sum |t|^2 over the samples idx (normalised targets):
    1 means no better than no closure, 0 exact."""
    torch = _torch()
    zero = torch.zeros(net.ncell * NOUT, dtype=torch.float32, device="cuda")
    num = den = 0.0
    for s in idx:
        net.forward(data.X[s], keep=False)
        net.loss.zero_()
        net._ck(net.lib.tcgpu_nn_mse(_p(net.out), _p(data.T[s]), None, net.ncell, NOUT, 16, _p(net.g[4]),
                                     _p(net.loss), None), "mse")
        torch.cuda.synchronize()
        num += net.loss.item()
        net.loss.zero_()
        net._ck(net.lib.tcgpu_nn_mse(_p(zero), _p(data.T[s]), None, net.ncell, NOUT, 16, _p(net.g[4]),
                                     _p(net.loss), None), "mse")
        torch.cuda.synchronize()
        den += net.loss.item()
    return num / den


def run_coarse(s, t_end: float, net: ClosureNet | None = None, in_scale=None, t_scale=None, max_steps: int = 100000,
               wall_model: WallModel | None = None, per_substep: bool = False):
    """Adaptive steps of the device-resident coarse solver s until its time
    reaches t_end, with the network's forcing when net is given: computed from
    the state at the start of each step and held over the step, or, with
    per_substep, computed again from the state at the start of every RK
    substep (the step then runs through the reference's stage entry points).
    Returns the times, the energy injection (inner-wall torque, the
    reference's estimator on this grid) after every step and, with
    wall_model, the wall model's torque after every step."""
    lib = s.lib
    st = stream_of(s)
    times, torque = [0.0], [s.diagnostics()["injection_u"]]
    wall = [wall_model.torque(s)] if wall_model is not None else None

    def forcing():
        s._check(lib.tcgpu_closure_input(C.byref(s.domain), C.byref(s.fluid), _d3(in_scale), NIN,
                                         _p(net.a[0])), "closure_input")
        net.forward(stream=st, keep=False)
        s._check(lib.tcgpu_set_forcing(C.byref(s.domain), C.byref(s.fluid), _p(net.out), NOUT, _d3(t_scale)),
                 "set_forcing")

    t = 0.0
    for _ in range(max_steps):
        if t >= t_end:
            break
        if net is not None and per_substep:
            dt = s.decide_dt()
            for rk in range(3):
                forcing()
                s.predict(rk, dt)
                s.compute_potential(rk, dt)
                s.correct_velocity(rk, dt)
                s.update_pressure(rk, dt)
            t += dt
        else:
            if net is not None:
                forcing()
            t += float(s.run(1)[0])
        times.append(t)
        torque.append(s.diagnostics()["injection_u"])
        if wall is not None:
            wall.append(wall_model.torque(s))
    if net is not None:
        s._check(lib.tcgpu_set_forcing(C.byref(s.domain), C.byref(s.fluid), None, NOUT, _d3((1, 1, 1))),
                 "set_forcing")
    if wall is not None:
        return np.asarray(times), np.asarray(torque), np.asarray(wall)
    return np.asarray(times), np.asarray(torque)


def time_average(times, values) -> float:
    """trapezoidal mean of values(times) over [times[0], times[-1]]"""
    t = np.asarray(times, dtype=np.float64)
    v = np.asarray(values, dtype=np.float64)
    return float(np.sum(0.5 * (v[1:] + v[:-1]) * np.diff(t)) / (t[-1] - t[0]))


def _main(argv=None) -> int:
    """python -m simpletcsolver_b200.closure [--grid NXxNYxNZ] [--iters N]:
    time the network's forward and backward passes on a synthetic input of a
    coarse grid (CUDA events on the stream the kernels run on)."""
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", default="64x256x128")
    ap.add_argument("--iters", type=int, default=10)
    args = ap.parse_args(argv)
    torch = _torch()
    grid = tuple(int(v) for v in args.grid.lower().split("x"))
    lib = abi.load()
    net = ClosureNet(lib, grid, seed=0)
    gen = torch.Generator(device="cuda").manual_seed(0)
    x = torch.randn(net.ncell * NIN, device="cuda", generator=gen).to(torch.bfloat16)
    tgt = torch.randn(net.ncell * NOUT, device="cuda", generator=gen)
    net.forward(x)
    net.backward(tgt, x=x)
    torch.cuda.synchronize()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    e[0].record()
    for _ in range(args.iters):
        net.forward(x)
    e[1].record()
    for _ in range(args.iters):
        net.backward(tgt, x=x)
    e[2].record()
    torch.cuda.synchronize()
    f_ms, b_ms = e[0].elapsed_time(e[1]) / args.iters, e[1].elapsed_time(e[2]) / args.iters
    flop = 2 * 27 * (4 * 32 + 32 * 32 + 32 * 32 + 32 * 3) * net.ncell
    print(f"grid {grid}: forward {f_ms:.3f} ms ({flop / f_ms / 1e9:.1f} TFLOP/s), backward {b_ms:.3f} ms")
    if lib.tcgpu_nn_status(1) != 0:
        print("a network kernel reported a wait that gave up")
        return 1
    return 0


if __name__ == "__main__":
    raise SystemExit(_main())
