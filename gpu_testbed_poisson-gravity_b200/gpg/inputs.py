"""Seeded synthetic patch inputs for the per-patch Poisson-gravity path.

The reference testbed fills its arrays with a power-law profile in
``Main.cpp:524-580`` (``Initialize``).  That form is singular at power index
2 (``Main.cpp:552``: A has (n-2) in its denominator), so this module uses the
gauge-fixed analytic potential

    phi(r) = 4 pi G rho0 r0^2 * ((r/r0)^(2-n) - 1) / ((2-n)(3-n))

which is continuous at n = 2 (where it becomes 4 pi G rho0 r0^2 ln(r/r0)) and
satisfies lap(phi) = 4 pi G rho0 (r/r0)^-n exactly.

Layout (all arrays C-contiguous, x fastest), matching the reference's array
shapes (``Header/Prototype.h:6-14``):

* ``rho``    [P][RHO_NXT][RHO_NXT][RHO_NXT]   fine density incl. RHO_GHOST_SIZE
* ``pot_in`` [P][POT_NXT][POT_NXT][POT_NXT]   coarse (2*dh) potential
* ``flu``    [P][5][8][8][8]                  density, px, py, pz, energy

Geometry: a box of 16^3 patches (128^3 fine cells, dh = 1) centred at
(64, 64, 64).  Patch p sits at patch coordinates (p % 16, p//16 % 16,
p//256 % 16); larger batches reuse positions with fresh noise.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

PATCH_SIZE = 8
NCOMP = 5
NEWTON_G = 1.0e-5
POI_COEFF = 4.0 * math.pi * NEWTON_G  # Main.cpp:184 (4*pi*NEWTON_G)
DH = 1.0                               # Makefile:47
DT = 1.0e-2                            # Makefile:48
BOX_PATCHES = 16
BOX_CENTRE = 0.5 * BOX_PATCHES * PATCH_SIZE

# Default SOR parameters, Main.cpp:1142-1157 (omega per ghost size 1..5).
SOR_OMEGA = {1: 1.49, 2: 1.57, 3: 1.62, 4: 1.65, 5: 1.69}
SOR_MIN_ITER = 10
SOR_MAX_ITER = {4: 60, 8: 100}         # keyed by sizeof(real)
# Default MG parameters, Main.cpp:1173-1223.
MG_MAX_ITER = {4: 10, 8: 20}
MG_TOL = {4: 1.0e-6, 8: 1.0e-15}
MG_NPRE = 3
MG_NPOST = 3


@dataclass(frozen=True)
class Geometry:
    """Per-patch array extents, Header/Macro.h:53-61."""

    ghost: int          # POT_GHOST_SIZE
    gra_ghost: int      # GRA_GHOST_SIZE

    @property
    def pot_int(self) -> int:
        return 0 if self.ghost == 0 else (self.ghost + 3) // 2

    @property
    def pot_nxt(self) -> int:
        return PATCH_SIZE // 2 + 2 * self.pot_int

    @property
    def rho_nxt(self) -> int:
        return PATCH_SIZE + 2 * (self.ghost - 1)

    @property
    def gra_nxt(self) -> int:
        return PATCH_SIZE + 2 * self.gra_ghost

    @property
    def cube(self) -> int:
        """Edge of the fine cube the solver works in (interior + 1 ghost layer)."""
        return PATCH_SIZE + 2 * self.ghost


def potential_profile(r, rho0, index, r0):
    """Gauge-fixed analytic potential of rho = rho0 (r/r0)^-index."""
    s = np.asarray(r, dtype=np.float64) / r0
    two_n = 2.0 - np.asarray(index, dtype=np.float64)
    ln_s = np.log(s)
    with np.errstate(divide="ignore", invalid="ignore"):
        general = np.expm1(two_n * ln_s) / (two_n * (3.0 - np.asarray(index, dtype=np.float64)))
    at_two = ln_s / (3.0 - np.asarray(index, dtype=np.float64))
    f = np.where(np.abs(two_n) < 1e-9, at_two, general)
    return POI_COEFF * rho0 * r0 * r0 * f


def _patch_corners(npatch: int) -> np.ndarray:
    p = np.arange(npatch, dtype=np.int64)
    pos = np.stack([p % BOX_PATCHES, (p // BOX_PATCHES) % BOX_PATCHES,
                    (p // BOX_PATCHES ** 2) % BOX_PATCHES], axis=1)
    return (pos * PATCH_SIZE).astype(np.float64)          # [P, 3] (x, y, z)


def _radius(corner, offset, n, spacing):
    """Radius of cell centres of an n^3 window starting `offset` fine cells
    below each patch corner, with cell size `spacing` fine cells."""
    idx = np.arange(n, dtype=np.float64) * spacing + 0.5 * spacing - offset
    x = corner[:, 0, None, None, None] + idx[None, None, None, :]
    y = corner[:, 1, None, None, None] + idx[None, None, :, None]
    z = corner[:, 2, None, None, None] + idx[None, :, None, None]
    c = BOX_CENTRE
    return np.sqrt((x - c) ** 2 + (y - c) ** 2 + (z - c) ** 2)


def make_patches(npatch: int, ghost: int, seed: int, *, gra_ghost: int = 1,
                 rho0=1.0, index=2.0, r0: float = 8.0, noise: float = 0.05,
                 dtype=np.float32, fluid: bool = True) -> dict:
    """Build one batch of patches.

    rho0 / index may be scalars or per-patch arrays.  The fluid density is the
    patch-interior part of the noisy density; velocities are N(0, 0.1) per
    component (momentum = density * velocity) and the energy is 1 + U(0, 0.1).
    All draws use numpy PCG64 seeded by ``seed``; values are generated in
    float64 and rounded once to ``dtype``.
    """
    if not 1 <= ghost <= 5:
        raise ValueError("ghost must be in 1..5")
    geo = Geometry(ghost, gra_ghost)
    rng = np.random.Generator(np.random.PCG64(seed))
    corner = _patch_corners(npatch)
    rho0 = np.broadcast_to(np.asarray(rho0, dtype=np.float64), (npatch,))
    index = np.broadcast_to(np.asarray(index, dtype=np.float64), (npatch,))
    bc = (slice(None), None, None, None)

    m = geo.rho_nxt
    r_f = _radius(corner, ghost - 1, m, 1.0)
    rho = rho0[bc] * (r_f / r0) ** (-index[bc])
    rho = rho * (1.0 + noise * rng.standard_normal(rho.shape))

    pn = geo.pot_nxt
    r_c = _radius(corner, 2 * geo.pot_int, pn, 2.0)
    pot = potential_profile(r_c, rho0[bc], index[bc], r0)

    out = {"rho": np.ascontiguousarray(rho.astype(dtype)),
           "pot_in": np.ascontiguousarray(pot.astype(dtype)),
           "geometry": geo}
    if fluid:
        lo = ghost - 1
        dens = rho[:, lo:lo + PATCH_SIZE, lo:lo + PATCH_SIZE, lo:lo + PATCH_SIZE]
        vel = 0.1 * rng.standard_normal((npatch, 3) + dens.shape[1:])
        eng = 1.0 + 0.1 * rng.random(dens.shape)
        flu = np.empty((npatch, NCOMP) + dens.shape[1:], dtype=np.float64)
        flu[:, 0] = dens
        flu[:, 1:4] = dens[:, None] * vel
        flu[:, 4] = eng
        out["flu"] = np.ascontiguousarray(flu.astype(dtype))
    return out


def mixed_ghost_assignment(npatch: int, seed: int,
                           fractions=(0.3, 0.3, 0.2, 0.1, 0.1)) -> np.ndarray:
    """Ghost size (1..5) per patch in the given proportions, seeded shuffle."""
    counts = np.floor(np.asarray(fractions) * npatch).astype(np.int64)
    counts[0] += npatch - counts.sum()
    g = np.repeat(np.arange(1, 6, dtype=np.int32), counts)
    rng = np.random.Generator(np.random.PCG64(seed))
    rng.shuffle(g)
    return g


def log_uniform(npatch: int, seed: int, lo: float = 1.0, decades: float = 4.0) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    return lo * 10.0 ** (decades * rng.random(npatch))
