"""Learned closure on the B200 against its CPU oracle (oracle/closure_ref.py).

The network kernels compute with BF16 operands and FP32 accumulation: FP32
outputs of BF16 inputs are held to 1e-5 relative, BF16 outputs (one rounding,
2^-8) to 1e-2, gradients through BF16 activations to 2e-2 relative L2. The
grid-side kernels are FP64 and held to round-off.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from oracle import closure_ref as cr
from oracle import tc_numpy as tn
from simpletcsolver_b200 import abi, closure, ic
from simpletcsolver_b200.solver import Solver
from tests._helpers import oracle_layout

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def _p(t):
    return C.c_void_p(t.data_ptr())


def _rel_max(a, b):
    return float((a - b).abs().max() / b.abs().max())


@pytest.mark.parametrize("grid", [(16, 32, 6), (64, 256, 32)])
@pytest.mark.parametrize("cinp,coutp,cin,cout", [(16, 32, 4, 32), (32, 32, 32, 32), (32, 16, 32, 3)])
def test_convolution_passes_match_cpu_oracle(lib, cinp, coutp, cin, cout, grid):
    """forward (linear and GELU epilogues), input and weight gradients of one
    layer, tensor-core kernels vs torch FP64 on the CPU. 16 x 32 x 6: one
    output plane per CTA; 64 x 256 x 32: about 14 planes per CTA, so the
    accumulator ring wraps, planes collect in the overflow blocks and CTA
    ranges cross column tiles."""
    torch = _torch()
    F = torch.nn.functional
    nx, ny, nz = grid
    g = torch.Generator().manual_seed(7)
    bf = lambda t: t.to(torch.bfloat16).to(torch.float64)
    x = torch.zeros(nz, ny, nx, cinp, dtype=torch.float64)
    x[..., :cin] = torch.randn(nz, ny, nx, cin, generator=g, dtype=torch.float64)
    x = bf(x)
    w = torch.randn(27, cout, cin, generator=g, dtype=torch.float64) * 0.2
    b = torch.zeros(coutp, dtype=torch.float64)
    b[:cout] = torch.randn(cout, generator=g, dtype=torch.float64) * 0.1
    wq = torch.zeros(27, coutp, cinp, dtype=torch.float64)
    wq[:, :cout, :cin] = bf(w)
    fwd = torch.zeros(27 * cinp * coutp, dtype=torch.bfloat16, device="cuda")
    bwd = torch.zeros_like(fwd)
    wd, bd = w.float().cuda(), b.float().cuda()
    assert lib.tcgpu_nn_pack_weights(_p(wd), cin, cout, cinp, coutp, _p(fwd), _p(bwd), None) == 0
    xd = x.to(torch.bfloat16).cuda()
    ref = cr.conv(x, wq, b)
    n = nx * ny * nz
    nout = min(cout, coutp)
    outf = torch.zeros(n * nout, device="cuda")
    assert lib.tcgpu_nn_conv3(1, cinp, coutp, nx, ny, nz, _p(xd), _p(fwd), _p(bd), None, None, None, _p(outf),
                              nout, None) == 0
    out = torch.zeros(n * coutp, dtype=torch.bfloat16, device="cuda")
    pre = torch.zeros_like(out)
    assert lib.tcgpu_nn_conv3(0, cinp, coutp, nx, ny, nz, _p(xd), _p(fwd), _p(bd), None, _p(out), _p(pre), None, 0,
                              None) == 0
    dy = bf(torch.randn(nz, ny, nx, coutp, generator=g, dtype=torch.float64))
    dy[..., cout:] = 0.0
    zs = bf(torch.randn(nz, ny, nx, cinp, generator=g, dtype=torch.float64))
    dyd, zsd = dy.to(torch.bfloat16).cuda(), zs.to(torch.bfloat16).cuda()
    dx = torch.zeros(n * cinp, dtype=torch.bfloat16, device="cuda")
    assert lib.tcgpu_nn_conv3(2, coutp, cinp, nx, ny, nz, _p(dyd), _p(bwd), None, _p(zsd), _p(dx), None, None, 0,
                              None) == 0
    ws = lib.tcgpu_nn_wgrad_workspace(nx, ny, nz, coutp)
    wsd = torch.zeros(ws // 4 + 4, device="cuda")
    dw = torch.zeros(27 * cout * cin, device="cuda")
    db = torch.zeros(cout, device="cuda")
    assert lib.tcgpu_nn_conv3_wgrad(cinp, coutp, cin, cout, nx, ny, nz, _p(xd), _p(dyd), _p(dw), _p(db), 0.0, _p(wsd),
                                    ws, None) == 0
    torch.cuda.synchronize()
    assert lib.tcgpu_nn_status(1) == 0
    got = outf.cpu().double().reshape(nz, ny, nx, nout)
    assert _rel_max(got, ref[..., :nout]) < 1e-5
    assert _rel_max(out.cpu().double().reshape(nz, ny, nx, coutp), F.gelu(ref, approximate="tanh")) < 1e-2
    assert _rel_max(pre.cpu().double().reshape(nz, ny, nx, coutp), ref) < 1e-2
    xr = torch.zeros_like(x, requires_grad=True)
    gx, = torch.autograd.grad(cr.conv(xr, wq), xr, dy)
    zz = zs.clone().requires_grad_(True)
    gz, = torch.autograd.grad(F.gelu(zz, approximate="tanh"), zz, torch.ones_like(zz))
    assert _rel_max(dx.cpu().double().reshape(nz, ny, nx, cinp), gx * gz) < 1e-2
    wr = torch.zeros(27, cout, cin, dtype=torch.float64, requires_grad=True)
    gw, = torch.autograd.grad(cr.conv(x[..., :cin], wr), wr, dy[..., :cout])
    assert _rel_max(dw.cpu().double().reshape(27, cout, cin), gw) < 1e-5
    assert _rel_max(db.cpu().double(), dy[..., :cout].sum(dim=(0, 1, 2))) < 1e-5


@pytest.mark.parametrize("grid", [(8, 16, 4), (64, 128, 64)])
def test_network_gradients_match_cpu_oracle(lib, grid):
    """loss and the gradients of all four layers through BF16 activations; at
    64 x 128 x 64 every convolution runs about 14 output planes per CTA"""
    torch = _torch()
    nx, ny, nz = grid
    net = closure.ClosureNet(lib, grid, seed=3, last_scale=1.0)
    g = torch.Generator().manual_seed(0)
    x = torch.zeros(nz, ny, nx, 16, dtype=torch.float64)
    x[..., :4] = torch.randn(nz, ny, nx, 4, generator=g, dtype=torch.float64)
    x = x.to(torch.bfloat16).to(torch.float64)
    tgt = torch.randn(nz, ny, nx, 3, generator=g, dtype=torch.float64)
    xd = x.to(torch.bfloat16).cuda().reshape(-1)
    net.loss.zero_()
    net.forward(xd)
    net.backward(tgt.float().cuda().reshape(-1), x=xd)
    torch.cuda.synchronize()
    P, G = net.params.cpu().double(), net.grads.cpu().double()
    params = []
    for li, (cin, _, cout, _) in enumerate(closure.LAYERS):
        w = P[net.woff[li]:net.woff[li] + 27 * cout * cin].reshape(27, cout, cin).to(torch.bfloat16).double()
        params.append((w, P[net.boff[li]:net.boff[li] + cout]))
    loss, og = cr.loss_and_grads(x[..., :4], tgt, params)
    assert abs(net.loss.item() - loss) < 1e-3 * loss
    for li, (cin, _, cout, _) in enumerate(closure.LAYERS):
        gw = G[net.woff[li]:net.woff[li] + 27 * cout * cin].reshape(27, cout, cin)
        gb = G[net.boff[li]:net.boff[li] + cout]
        assert float((gw - og[li][0]).norm() / og[li][0].norm()) < 2e-2, li
        assert float((gb - og[li][1]).norm() / og[li][1].norm()) < 2e-2, li


def test_adam_matches_cpu_oracle(lib):
    torch = _torch()
    rng = np.random.default_rng(1)
    p = rng.standard_normal(1000)
    m = np.zeros(1000)
    v = np.zeros(1000)
    pd = torch.tensor(p, dtype=torch.float32, device="cuda")
    md, vd = torch.zeros_like(pd), torch.zeros_like(pd)
    for step in range(1, 6):
        gr = rng.standard_normal(1000)
        p, m, v = cr.adam(p, gr, m, v, step)
        gd = torch.tensor(gr, dtype=torch.float32, device="cuda")
        assert lib.tcgpu_nn_adam(_p(pd), _p(gd), _p(md), _p(vd), 1000, 1e-3, 0.9, 0.999, 1e-8, step, None) == 0
    torch.cuda.synchronize()
    assert np.abs(pd.cpu().numpy() - p).max() < 1e-6


def _three_solvers(lib, tmp_path, case):
    d0 = ic.write_ic(case, str(tmp_path / "fine"))
    dc = closure.write_coarse_ic(case, str(tmp_path / "coarse"))
    cc = closure.coarse_case(case)
    out = []
    for d, cs in ((d0, case), (dc, cc), (dc, cc)):
        s = Solver.from_ic(d, case=cs, lib=lib)
        closure.resident(s)
        out.append(s)
    return d0, cc, out


def test_restriction_matches_oracle_and_stays_divergence_free(lib, tmp_path):
    """tcgpu_coarsen against the numpy restriction to round-off; the coarse
    field of a divergence-free fine field is divergence-free"""
    case = ic.taylor_couette(32, 64, 32, 3400.0)
    d0, cc, (fine, ca, cb) = _three_solvers(lib, tmp_path, case)
    try:
        fine.run(2)
        fine.pull()
        assert lib.tcgpu_coarsen(C.byref(fine.domain), C.byref(fine.fluid), C.byref(ca.domain),
                                 C.byref(ca.fluid)) == 0
        ca.pull()
        d = tn.load_domain(d0)
        ref = cr.restrict({n: oracle_layout(n, fine.field(n)) for n in ("ux", "uy", "uz", "t", "p")}, d)
        for n in ("ux", "uy", "uz", "t", "p"):
            g = ca.field(n)[1:-1, 1:-1]
            g = g[:, :, :cc.nx] if n == "ux" else g[:, :, 1:cc.nx + 1]
            assert np.abs(g - ref[n]).max() < 1e-13 * max(np.abs(ref[n]).max(), 1.0), n
        assert fine.diagnostics()["divmax"] < 1e-12
        assert ca.diagnostics()["divmax"] < 1e-12
    finally:
        for s in (fine, ca, cb):
            s.release()


def test_forcing_enters_the_explicit_terms(lib, tmp_path):
    """a zero forcing changes nothing (bit for bit); a uniform axial forcing
    f0 raises the volume mean of uz by f0 dt over one step (explicit diffusion:
    up to the wall shear it adds within the step, below 1%)"""
    torch = _torch()
    case = ic.taylor_couette(8, 16, 8, 500.0, implicit=(False, False, False))
    d0 = ic.write_ic(case, str(tmp_path / "ic"))
    n = case.nx * case.ny * case.nz

    def one_step(frc):
        s = Solver.from_ic(d0, case=case, lib=lib)
        try:
            closure.resident(s)
            if frc is not None:
                buf = torch.tensor(frc, dtype=torch.float32, device="cuda")
                assert lib.tcgpu_set_forcing(C.byref(s.domain), C.byref(s.fluid), _p(buf), 3,
                                             (C.c_double * 3)(1, 1, 1)) == 0
            dt = s.run(1)[0]
            s.pull()
            return dt, {k: s.field(k).copy() for k in ("ux", "uy", "uz", "t", "p")}
        finally:
            s.release()

    dt0, a = one_step(None)
    dt1, b = one_step(np.zeros((n, 3)))
    assert dt0 == dt1
    for k in a:
        np.testing.assert_array_equal(a[k], b[k])
    f0 = 1e-3
    fr = np.zeros((n, 3))
    fr[:, 2] = f0
    dt2, c = one_step(fr)
    w = tn.load_domain(d0).jdxc[1:case.nx + 1]
    dm = c["uz"][1:-1, 1:-1, 1:-1] - a["uz"][1:-1, 1:-1, 1:-1]
    shift = (dm * w).sum() / (w.sum() * case.ny * case.nz)
    assert abs(shift / (f0 * dt2) - 1.0) < 1e-2


def test_trained_closure_beats_no_closure_on_held_out_pairs(lib, tmp_path):
    """the 64x128x64 Taylor-Couette run restricted to 16x32x16: 64 training
    pairs, every 4th held out; after 80 epochs the network removes at least
    20% of the closure error (sum |f - t|^2 / sum |t|^2, 1 = no closure) on
    the held-out pairs and 30% on the training pairs"""
    case = ic.taylor_couette(64, 128, 64, 3400.0)
    _, cc, (fine, ca, cb) = _three_solvers(lib, tmp_path, case)
    try:
        fine.run(50)
        data, _ = closure.generate(fine, ca, cb, 64, 2, in_scale=(0.05, 1.0, 0.05))
        train = [s for s in range(64) if s % 4]
        held = [s for s in range(64) if s % 4 == 0]
        net = closure.ClosureNet(lib, (cc.nx, cc.ny, cc.nz), seed=0)
        before = closure.relative_error(net, data, held)
        hist = closure.train(net, data, train, epochs=80, batch=8, lr=2e-3)
        assert hist[-1] < hist[0]
        assert closure.relative_error(net, data, train) < 0.7
        after = closure.relative_error(net, data, held)
        assert after < 0.8 and after < before
        assert lib.tcgpu_nn_status(1) == 0
    finally:
        for s in (fine, ca, cb):
            s.release()


def test_wall_model_reproduces_the_injection_formula_and_learns(lib, tmp_path):
    """The wall model's per-face injection (injection.c:55-73 with the wall
    values of lyx.c and lxy.c) summed over the fine wall equals the fine
    solver's own energy injection; a model fitted on restricted/fine pairs
    predicts the fine first-cell velocity of held-out pairs better than the
    coarse first-cell value itself, and the radial slab entry point returns
    the device field's values."""
    case = ic.taylor_couette(64, 128, 64, 3400.0)
    _, cc, (fine, ca, cb) = _three_solvers(lib, tmp_path, case)
    try:
        fine.run(50)
        # slab against the pulled field
        fine.pull(abi.UY)
        slab = fine.radial_slab("uy", 0, 3)
        np.testing.assert_array_equal(slab, fine.field("uy")[1:-1, 1:-1, 0:3])
        data, _ = closure.generate(fine, ca, cb, 16, 2, in_scale=(0.05, 1.0, 0.05))
        train = [s for s in range(16) if s % 4]
        held = [s for s in range(16) if s % 4 == 0]
        wm = closure.WallModel.fit(data, train, fine, ca)
        got = closure.WallModel.fine_injection(wm, fine.radial_slab("uy", 1, 1))
        ref = fine.diagnostics()["injection_u"]
        assert abs(got - ref) <= 1e-11 * abs(ref)
        for q in held:
            tgt = closure.block_mean(data.wall_y[q], ca).ravel()
            err_model = np.sqrt(np.mean((wm.predict(data.wall_x[q]) - tgt) ** 2))
            err_raw = np.sqrt(np.mean((data.wall_x[q][:, :, 0].ravel() - tgt) ** 2))
            assert err_model < 0.5 * err_raw
    finally:
        for s in (fine, ca, cb):
            s.release()
