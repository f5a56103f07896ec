"""CPU oracle of the learned initial-guess network.  TEST INFRASTRUCTURE ONLY.

The reference has no learned component; this restates, in float64 numpy, the
network the library's tensor-core kernels compute (include/gpg.h, gpg_net_*),
rounding to bfloat16 exactly where the kernels store bfloat16, so that forward
activations and parameter gradients can be checked against the GPU.

Network (ghost size 1 patches, on the 10^3 solver cube, "same" padding):
  input  X0 [v][8]: 0 = Const*rho / s on interior cells, 1 = interpolated coarse
         potential / s on the ghost shell, 2 = interior mask, 3..7 = 0
         (s = max |potential| over the shell of the patch)
  L1 conv 3^3  8 -> 32, ReLU;  L2, L3 conv 3^3 32 -> 32, ReLU;
  L4 conv 3^3 32 -> 16 (output channel 0 is used), linear, float32
  guess = L4[.., 0] * s on the 8^3 interior
  loss  = mean over interior cells of (L4[.., 0] - phi_target / s)^2
Weights W[l] have shape [27][cin][cout] (tap = (dz+1)*9 + (dy+1)*3 + (dx+1)).
"""
from __future__ import annotations

import numpy as np

N = 10          # cube edge (ghost size 1)
CH = (8, 32, 32, 32, 16)


def bf16(a):
    """Round float values to bfloat16 (round to nearest even), returned as float64."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def taps():
    out = []
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                out.append((dz, dy, dx))
    return out


def shift(x, dz, dy, dx):
    """y[p, z, y, x, c] = x[p, z+dz, y+dy, x+dx, c], zero outside the cube."""
    y = np.zeros_like(x)
    zs = slice(max(0, -dz), N - max(0, dz))
    ys = slice(max(0, -dy), N - max(0, dy))
    xs = slice(max(0, -dx), N - max(0, dx))
    zt = slice(max(0, dz), N - max(0, -dz))
    yt = slice(max(0, dy), N - max(0, -dy))
    xt = slice(max(0, dx), N - max(0, -dx))
    y[:, zs, ys, xs, :] = x[:, zt, yt, xt, :]
    return y


def conv(x, w, b):
    """x [P][N][N][N][cin], w [27][cin][cout], b [cout] -> [P][N][N][N][cout] (float64)."""
    out = np.zeros(x.shape[:4] + (w.shape[2],))
    for t, (dz, dy, dx) in enumerate(taps()):
        out += shift(x, dz, dy, dx) @ w[t]
    return out + b


def conv_t(g, w):
    """Adjoint of conv wrt its input: g [..][cout] -> [..][cin]."""
    out = np.zeros(g.shape[:4] + (w.shape[1],))
    for t, (dz, dy, dx) in enumerate(taps()):
        out += shift(g, -dz, -dy, -dx) @ w[t].T
    return out


def conv_w(x, g):
    """Weight gradient: sum_v x[v + off(t)] g[v] -> [27][cin][cout]."""
    out = np.zeros((27, x.shape[-1], g.shape[-1]))
    gf = g.reshape(-1, g.shape[-1])
    for t, (dz, dy, dx) in enumerate(taps()):
        out[t] = shift(x, dz, dy, dx).reshape(-1, x.shape[-1]).T @ gf
    return out


def make_input(rho, cube, const):
    """rho [P][8][8][8], cube [P][10][10][10] (interpolated coarse potential) ->
    (X0 [P][10][10][10][8] bf16-rounded, s [P])."""
    p = rho.shape[0]
    shell = np.ones((N, N, N), dtype=bool)
    shell[1:-1, 1:-1, 1:-1] = False
    s = np.abs(cube.astype(np.float64)[:, shell]).max(axis=1)
    s = np.where(s > 0, s, 1.0).astype(np.float32).astype(np.float64)
    x = np.zeros((p, N, N, N, 8))
    x[:, 1:-1, 1:-1, 1:-1, 0] = (np.float32(const) * rho.astype(np.float32)).astype(np.float64) / s[:, None, None, None]
    x[:, :, :, :, 1] = np.where(shell, cube.astype(np.float64) / s[:, None, None, None], 0.0)
    x[:, 1:-1, 1:-1, 1:-1, 2] = 1.0
    return bf16(x), s


def forward(x0, w, b):
    """Returns activations [x0, a1, a2, a3] (bf16-rounded) and y4 (float64)."""
    acts = [x0]
    a = x0
    for l in range(3):
        a = bf16(np.maximum(conv(a, bf16(w[l]), b[l]), 0.0))
        acts.append(a)
    y4 = conv(a, bf16(w[3]), b[3])
    return acts, y4


def loss_and_grads(x0, w, b, target, s):
    """target [P][8][8][8] interior potential.  Returns (loss, dW list, db list)."""
    acts, y4 = forward(x0, w, b)
    p = x0.shape[0]
    t = target.astype(np.float64) / s[:, None, None, None]
    diff = y4[:, 1:-1, 1:-1, 1:-1, 0] - t
    cnt = p * 512
    loss = float((diff ** 2).sum() / cnt)
    g = np.zeros(y4.shape)
    g[:, 1:-1, 1:-1, 1:-1, 0] = 2.0 * diff / cnt
    g = bf16(g)
    dws, dbs = [None] * 4, [None] * 4
    for l in (3, 2, 1, 0):
        dws[l] = conv_w(acts[l], g)
        dbs[l] = g.reshape(-1, g.shape[-1]).sum(axis=0)
        if l > 0:
            g = bf16(conv_t(g, bf16(w[l])) * (acts[l] > 0))
    return loss, dws, dbs
