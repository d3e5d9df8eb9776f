"""Synthetic lattices for the benchmark configurations (seeded, deterministic).

Each generator returns an (R, C) grid of the reference's InputNodeType codes
(llalbm/src/utils/aliases.hpp:41-48); row index i grows downwards (row 0 is the
top of the domain), column index j grows to the right, as in the reference.

  cavity_types(129)            config 1: lid-driven cavity (= test/assets/lid-lattice.txt)
  cylinder_types()             config 2: 1024 x 256 channel with a radius-20 cylinder
  porous_types(4096, 4096)     config 3: random non-overlapping discs, 30 % solid
"""
from __future__ import annotations

import numpy as np

FLUID, SOLID, BOUNDARY, INLET, OUTLET, OBSTACLE = range(6)


def cavity_types(n: int) -> np.ndarray:
    """Lid-driven cavity: perimeter walls, lid (inlet) on row 0, columns 1..n-2."""
    t = np.zeros((n, n), dtype=np.uint8)
    t[0, :] = t[-1, :] = t[:, 0] = t[:, -1] = BOUNDARY
    t[0, 1:-1] = INLET
    return t


def channel_types(R: int, C: int, discs=(), outlet: bool = True) -> np.ndarray:
    """Channel: walls on rows 0 and R-1, inlet on column 0 and outlet on column
    C-1 (rows 1..R-2), obstacle discs (ci, cj, r) with |d|^2 <= r^2."""
    t = np.zeros((R, C), dtype=np.uint8)
    t[0, :] = t[-1, :] = BOUNDARY
    t[1:-1, 0] = INLET
    t[1:-1, -1] = OUTLET if outlet else BOUNDARY
    ii, jj = np.mgrid[0:R, 0:C]
    for ci, cj, r in discs:
        t[((ii - ci) ** 2 + (jj - cj) ** 2 <= r * r) & (t == FLUID)] = OBSTACLE
    return t


def cylinder_types(R: int = 256, C: int = 1024, x0: int = 200, y0: int = 131, r: int = 20) -> np.ndarray:
    """Channel with a staircase cylinder (x - x0)^2 + (y - y0)^2 <= r^2, where
    x = j and y = R - 1 - i points up (the direction of u_y)."""
    t = channel_types(R, C)
    ii, jj = np.mgrid[0:R, 0:C]
    y = R - 1 - ii
    t[((jj - x0) ** 2 + (y - y0) ** 2 <= r * r) & (t == FLUID)] = OBSTACLE
    return t


def porous_types(R: int, C: int, fraction: float = 0.30, rmin: int = 3, rmax: int = 12,
                 seed: int = 20261203, gap: int = 1, margin: int = 2) -> np.ndarray:
    """Random porous channel: discs with integer radius uniform in [rmin, rmax]
    and centres uniform over the lattice, placed until the solid fraction of the
    grid reaches `fraction`.  A disc is rejected if any of its nodes, grown by
    `gap`, touches an earlier disc, or if it comes within `margin` nodes of the
    walls, inlet or outlet.  numpy PCG64 with a fixed seed."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t = channel_types(R, C)
    solid = np.zeros((R, C), dtype=bool)
    target = fraction * R * C
    count = 0
    offs = {}
    while count < target:
        r = int(rng.integers(rmin, rmax + 1))
        ci = int(rng.integers(0, R))
        cj = int(rng.integers(0, C))
        lo = margin + r + 1
        if ci < lo or ci > R - 1 - lo or cj < lo or cj > C - 1 - lo:
            continue
        if r not in offs:
            a = np.arange(-r - gap, r + gap + 1)
            di, dj = np.meshgrid(a, a, indexing="ij")
            grown = di * di + dj * dj <= (r + gap) * (r + gap)
            disc = di * di + dj * dj <= r * r
            offs[r] = (di[grown], dj[grown], di[disc], dj[disc])
        gi, gj, di, dj = offs[r]
        if solid[ci + gi, cj + gj].any():
            continue
        solid[ci + di, cj + dj] = True
        count += len(di)
    t[solid] = OBSTACLE
    return t


def parabolic_u(i: int, umax: float, i0: int, i1: int) -> float:
    """Poiseuille inlet profile across rows i0..i1 with half-way walls:
    4 umax yy (H - yy) / H^2, yy = (i - i0) + 0.5, H = i1 - i0 + 1."""
    H = float(i1 - i0 + 1)
    yy = float(i - i0) + 0.5
    return 4.0 * umax * yy * (H - yy) / (H * H)


def channel_discs_types(R: int, C: int, n_discs: int, rng: np.random.Generator) -> np.ndarray:
    """Channel with n_discs non-overlapping random discs (radius 3..max(3, min(R, C) // 8),
    kept one node clear of each other and two nodes clear of walls, inlet and outlet)."""
    t = channel_types(R, C)
    solid = np.zeros((R, C), dtype=bool)
    rmax = max(3, min(R, C) // 8)
    placed, tries = 0, 0
    ii, jj = np.mgrid[0:R, 0:C]
    while placed < n_discs and tries < 200 * max(n_discs, 1):
        tries += 1
        r = int(rng.integers(3, rmax + 1))
        ci, cj = int(rng.integers(0, R)), int(rng.integers(0, C))
        lo = r + 3
        if ci < lo or ci > R - 1 - lo or cj < lo or cj > C - 1 - lo:
            continue
        grown = (ii - ci) ** 2 + (jj - cj) ** 2 <= (r + 1) ** 2
        if solid[grown].any():
            continue
        solid[(ii - ci) ** 2 + (jj - cj) ** 2 <= r * r] = True
        placed += 1
    t[solid] = OBSTACLE
    return t


def batch_problems(n: int = 256, seed: int = 20261204, max_nx: int = 1024):
    """Config 4: n independent problems.  nx (columns) uniform in {64, 96, ...,
    max_nx}, aspect ratio a uniform in [1, 4], ny = round(nx * a) rows; half
    lid-driven cavities (lid u_x uniform in [0.02, 0.1]), half channels with 0-8
    random discs (Zou-He inlet u_x uniform in [0.02, 0.1], Zou-He pressure outlet
    rho = 1); tau uniform in [0.55, 1.5]; BGK or TRT (magic parameter 1/4) with
    probability 1/2 each.  numpy PCG64 with a fixed seed.  Each problem is a dict
    with `types` generated lazily by `make_types()`."""
    rng = np.random.Generator(np.random.PCG64(seed))
    sizes = np.arange(64, max_nx + 1, 32)
    out = []
    for q in range(n):
        nx = int(rng.choice(sizes))
        a = float(rng.uniform(1.0, 4.0))
        ny = int(round(nx * a))
        cavity = q % 2 == 0
        u = float(rng.uniform(0.02, 0.1))
        tau = float(rng.uniform(0.55, 1.5))
        trt = bool(rng.integers(0, 2))
        n_discs = 0 if cavity else int(rng.integers(0, 9))
        disc_seed = int(rng.integers(0, 2**31))
        tau_odd = 0.25 * (1.0 / (tau - 0.5)) + 0.5
        def make(ny=ny, nx=nx, cavity=cavity, n_discs=n_discs, disc_seed=disc_seed):
            if cavity:
                t = np.zeros((ny, nx), dtype=np.uint8)
                t[0, :] = t[-1, :] = t[:, 0] = t[:, -1] = BOUNDARY
                t[0, 1:-1] = INLET
                return t
            return channel_discs_types(ny, nx, n_discs, np.random.Generator(np.random.PCG64(disc_seed)))
        out.append(dict(rows=ny, cols=nx, kind="cavity" if cavity else "channel", u=u, tau=tau, trt=trt,
                        tau_odd=tau_odd, n_discs=n_discs, make_types=make,
                        outlet_bc=0 if cavity else 2))
    return out
