"""CPU restatement of the learned-closure pieces (no counterpart in the
reference): the 4x restriction of a fine state, the network input, the
3x3x3 convolutional network with its gradients, and Adam.

TEST INFRASTRUCTURE ONLY: the oracle that the CUDA closure kernels are checked
against (tests/ only). FP64: numpy for the grid side, torch on the CPU for the
network (autograd gives the reference gradients).

Conventions shared with the CUDA side: activations [k][j][i][c] over the
interior cells of the coarse grid; weights w[t][co][ci] with
t = 9 (dz+1) + 3 (dy+1) + (dx+1); convolution = cross-correlation, zero padding
in x (radial), periodic in y and z; GELU in its tanh form.
"""
from __future__ import annotations

import numpy as np

R = 4


def restrict(fine: dict, d) -> dict:
    """Coarse interior values (numpy [k][j][i], i from 1) of the fine fields
    (oracle layout, tc_numpy: A[k, j, i] with halos; ux with its unused i = 0
    column): ux at coarse face I = mean over the R^2 fine faces 4 (I-1) + 1;
    uy at coarse y-face J weighted by J/hy of the fine cells; uz at coarse
    z-face K weighted by J/hz; t and p volume (J) weighted."""
    nx, ny, nz = d.nx // R, d.ny // R, d.nz // R
    out = {}
    ux = fine["ux"]
    faces = ux[1:d.nz + 1, 1:d.ny + 1, 1:d.nx + 1:R]             # fine faces 1, 5, ... (nx of them)
    out["ux"] = faces.reshape(nz, R, ny, R, nx).mean(axis=(1, 3))
    out["ux"][:, :, 0] = 0.0
    i = np.arange(1, d.nx + 1)
    wy = d.jdxc[i] / d.hyxc[i]
    wz = d.jdxc[i] / d.hz
    wv = d.jdxc[i]
    uy = fine["uy"][1:d.nz + 1, 1:d.ny + 1:R, 1:d.nx + 1]        # fine y-faces 1, 5, ...
    out["uy"] = ((uy * wy).reshape(nz, R, ny, nx, R).sum(axis=(1, 4))
                 / (R * wy.reshape(nx, R).sum(axis=1))[None, None, :])
    uz = fine["uz"][1:d.nz + 1:R, 1:d.ny + 1, 1:d.nx + 1]
    out["uz"] = ((uz * wz).reshape(nz, ny, R, nx, R).sum(axis=(2, 4))
                 / (R * wz.reshape(nx, R).sum(axis=1))[None, None, :])
    for n in ("t", "p"):
        a = fine[n][1:d.nz + 1, 1:d.ny + 1, 1:d.nx + 1]
        out[n] = ((a * wv).reshape(nz, R, ny, R, nx, R).sum(axis=(1, 3, 5))
                  / (R * R * wv.reshape(nx, R).sum(axis=1))[None, None, :])
    return out


def network_input(ux, uy, uz, scale) -> np.ndarray:
    """[k][j][i][16]: ux averaged to the centre / scale[0], uy / scale[1],
    uz / scale[2], radial index coordinate 2 (i + 1/2) / nx - 1, zeros.
    ux: faces 1..nx+1 as [k][j][nx+1]; uy, uz: centres [k][j][nx]."""
    nz, ny, nx = uy.shape
    x = np.zeros((nz, ny, nx, 16))
    x[..., 0] = 0.5 * (ux[..., :-1] + ux[..., 1:]) / scale[0]
    x[..., 1] = uy / scale[1]
    x[..., 2] = uz / scale[2]
    x[..., 3] = (2.0 * (np.arange(nx) + 0.5) / nx - 1.0)[None, None, :]
    return x


def conv(x, w, b=None):
    """torch CPU: x [k][j][i][cin], w [27][cout][cin] -> [k][j][i][cout]."""
    import torch
    F = torch.nn.functional
    xt = x.permute(3, 0, 1, 2)[None]
    xt = F.pad(xt, (0, 0, 1, 1, 1, 1), mode="circular")
    xt = F.pad(xt, (1, 1, 0, 0, 0, 0))
    co, ci = w.shape[1], w.shape[2]
    y = F.conv3d(xt, w.reshape(3, 3, 3, co, ci).permute(3, 4, 0, 1, 2))[0].permute(1, 2, 3, 0)
    return y if b is None else y + b


def network(x, params):
    """params: [(w, b)] of the four layers (torch tensors); GELU (tanh form)
    after the first three."""
    import torch
    F = torch.nn.functional
    h = x
    for li, (w, b) in enumerate(params):
        h = conv(h, w, b)
        if li < len(params) - 1:
            h = F.gelu(h, approximate="tanh")
    return h


def loss_and_grads(x, target, params):
    """mean squared error of the network output (channels of target) and its
    gradients with respect to every (w, b), FP64 on the CPU."""
    import torch
    ps = [(w.clone().requires_grad_(True), b.clone().requires_grad_(True)) for (w, b) in params]
    out = network(x, ps)[..., :target.shape[-1]]
    loss = ((out - target) ** 2).mean()
    flat = [t for pair in ps for t in pair]
    grads = torch.autograd.grad(loss, flat)
    return loss.item(), [(grads[2 * i], grads[2 * i + 1]) for i in range(len(ps))]


def adam(p, g, m, v, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    """one Adam step (Kingma and Ba 2015) in numpy FP64; returns p, m, v"""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    p = p - lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return p, m, v
