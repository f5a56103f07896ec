"""CPU restatement of the learned linear correction.  TEST INFRASTRUCTURE ONLY.

The correction has no counterpart in the reference; what it builds on does:
the interpolated start (CPU_PoissonSolver_SOR.cpp:110-174, via the C oracle's
interp_cube) and the SOR residual expression (CPU_PoissonSolver_SOR.cpp:
232-237).  The library's kernel (csrc/lin_sor.cuh) must reproduce:

* ``residual``   r0 on the 8^3 interior, FP32, the residual's operand order;
* ``fold``       per mirror orbit a length-8 Walsh-Hadamard transform (FP32,
                 stages x, y, z), blocks re-indexed into their class's axes;
* ``apply``      block b times W[class(b)] with BF16 operands (FP64 sums here;
                 the tensor cores sum in FP32), then the unfold (FP32) and
                 the FP32 add to the interpolated start;
* ``features``   the training input: the folded residual, scaled by the
                 power of two of the patch's largest interpolated potential;
* ``targets``    the folded (target - start) / 8, scaled the same way;
* ``gradients``  the training loss and its gradient (FP64).

``green_params`` gives the exact correction: the block form of minus the
inverse 7-point Laplacian of the 8^3 interior with zero boundary values.
Only tests/, __graft_entry__.smoke() and bench.py's CPU leg use this module.
"""
from __future__ import annotations

import numpy as np

K = 64


def perm_of(b: int) -> int:
    return 1 if b == 2 else (2 if b in (4, 6) else (3 if b == 5 else 0))


def class_of(b: int) -> int:
    return bin(b).count("1")


def perm_orbit(o: int, t: int) -> int:
    k, j, i = o >> 4, (o >> 2) & 3, o & 3
    if t == 0:
        return o
    if t == 1:
        return (k << 4) | (i << 2) | j
    if t == 2:
        return (i << 4) | (j << 2) | k
    return (j << 4) | (k << 2) | i


def orbit_cell(o: int, s: int) -> int:
    k, j, i = o >> 4, (o >> 2) & 3, o & 3
    z = 7 - k if s & 4 else k
    y = 7 - j if s & 2 else j
    x = 7 - i if s & 1 else i
    return (z * 8 + y) * 8 + x


# [64][8] interior index of orbit o's image s; [8][64] class-axis position
CELL = np.array([[orbit_cell(o, s) for s in range(8)] for o in range(K)])
PERM = np.array([[perm_orbit(o, perm_of(b)) for o in range(K)] for b in range(8)])


def hadamard8(a):
    """In place over the last axis (length 8), FP32 or FP64 as given:
    out[b] = sum_s (-1)^popcount(b & s) in[s]; stages x, y, z."""
    a = a.copy()
    hb = 1
    while hb < 8:
        for i in range(8):
            if not i & hb:
                p, q = a[..., i].copy(), a[..., i | hb].copy()
                a[..., i] = p + q
                a[..., i | hb] = p - q
        hb <<= 1
    return a


def residual(cube, rho, cnst):
    """r0 [P][512] of interpolated cubes [P][10][10][10] (FP32):
    ((((((z+ + z-) + y+) + y-) + x+) + x-) - 6 phi) - cnst*rho."""
    c = np.asarray(cube, dtype=np.float32)
    f32 = np.float32
    s = c[:, 2:, 1:-1, 1:-1] + c[:, :-2, 1:-1, 1:-1]
    s = s + c[:, 1:-1, 2:, 1:-1]
    s = s + c[:, 1:-1, :-2, 1:-1]
    s = s + c[:, 1:-1, 1:-1, 2:]
    s = s + c[:, 1:-1, 1:-1, :-2]
    r = (s - f32(6) * c[:, 1:-1, 1:-1, 1:-1]) - f32(cnst) * np.asarray(rho, dtype=np.float32)
    return r.reshape(c.shape[0], 512)


def fold(x):
    """[P][512] (natural interior order) -> [P][8][64] (class axes), same dtype."""
    h = hadamard8(x[:, CELL])            # [P][64 orbits][8 blocks]
    out = np.empty((x.shape[0], 8, K), dtype=x.dtype)
    for b in range(8):
        out[:, b, PERM[b]] = h[:, :, b]
    return out


def unfold(v):
    """[P][8][64] (class axes) -> [P][512] natural order, FP32 stages."""
    nat = np.empty((v.shape[0], K, 8), dtype=v.dtype)
    for b in range(8):
        nat[:, :, b] = v[:, b, PERM[b]]
    d = hadamard8(nat)                   # [P][64 orbits][8 images]
    out = np.empty((v.shape[0], 512), dtype=v.dtype)
    out[:, CELL] = d
    return out


def bf16(a):
    """Round FP32 to the nearest BF16 (ties to even), returned as FP64."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def apply(w, u):
    """v [P][8][64] FP32 = W[class(b)] u_b with BF16-rounded operands."""
    wq = bf16(np.asarray(w, dtype=np.float32).reshape(4, K, K))
    uq = bf16(u)
    v = np.empty(u.shape, dtype=np.float64)
    for b in range(8):
        v[:, b] = uq[:, b] @ wq[class_of(b)].T
    return v.astype(np.float32)


def learned_start(w, cube, rho, cnst):
    """Interior start [P][8][8][8]: interpolated cube interior + correction."""
    u = fold(residual(cube, rho, cnst))
    d = unfold(apply(w, u))
    interior = np.asarray(cube, dtype=np.float32)[:, 1:-1, 1:-1, 1:-1].reshape(-1, 512)
    return (interior + d).reshape(-1, 8, 8, 8)


FEATURE_GAIN = 17


def feature_scale(cube):
    """[P] the power of two 2^(17 - e) with max|interpolated interior| = m 2^e,
    m in [0.5, 1) (e = 0 for an all-zero interior), FP32."""
    m = np.abs(np.asarray(cube, dtype=np.float32)[:, 1:-1, 1:-1, 1:-1]).reshape(len(cube), -1).max(1)
    ex = np.where(m > 0, np.frexp(m.astype(np.float64))[1], 0)
    return np.ldexp(1.0, FEATURE_GAIN - ex).astype(np.float32)


def features(cube, rho, cnst):
    """The training input u [P][8][64]: the folded residual, scaled."""
    return feature_scale(cube)[:, None, None] * fold(residual(cube, rho, cnst))


def targets(cube, target):
    """The training target t [P][8][64]: folded (target - interpolated
    interior) / 8, scaled like the features (FP32)."""
    interior = np.asarray(cube, dtype=np.float32)[:, 1:-1, 1:-1, 1:-1].reshape(-1, 512)
    d = np.asarray(target, dtype=np.float32).reshape(-1, 512) - interior
    return feature_scale(cube)[:, None, None] * (np.float32(0.125) * fold(d))


def gradients(w, u, t):
    """(loss, grad [4][64][64]) in FP64 of the training objective: the mean of
    e^2 over patches, blocks and rows, e = W[class] u - t."""
    w = np.asarray(w, dtype=np.float64).reshape(4, K, K)
    u = np.asarray(u, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    v = np.empty_like(u)
    for b in range(8):
        v[:, b] = u[:, b] @ w[class_of(b)].T
    e = v - t
    n = u.shape[0] * 512
    grad = np.zeros((4, K, K))
    for b in range(8):
        grad[class_of(b)] += e[:, b].T @ u[:, b]
    return float((e ** 2).sum() / n), grad * (2.0 / n)


def laplacian_interior() -> np.ndarray:
    """7-point Laplacian of the 8^3 interior with zero boundary values."""
    L = np.zeros((512, 512))
    for z in range(8):
        for y in range(8):
            for x in range(8):
                r = (z * 8 + y) * 8 + x
                L[r, r] = -6.0
                for dz, dy, dx in ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)):
                    zz, yy, xx = z + dz, y + dy, x + dx
                    if 0 <= zz < 8 and 0 <= yy < 8 and 0 <= xx < 8:
                        L[r, (zz * 8 + yy) * 8 + xx] = 1.0
    return L


def green_params() -> np.ndarray:
    """W[4][64][64] (FP64) of the exact correction delta = -L^-1 r0: for each
    class, v_b = fold(-L^-1 unfold(e_k) / 8) / 8 column by column of its
    representative block (b = 0, 1, 3, 7)."""
    G = -np.linalg.inv(laplacian_interior())
    w = np.zeros((4, K, K))
    for c, b in enumerate((0, 1, 3, 7)):
        u = np.zeros((K, 8, K))
        u[np.arange(K), b, np.arange(K)] = 1.0
        r0 = unfold(u) / 8.0
        v = fold(r0 @ G.T) / 8.0
        w[c] = v[:, b, :].T
    return w
