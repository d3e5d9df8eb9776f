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


def serve_requests(n: int = 96, seed: int = 20261205, side_min: int = 128, side_max: int = 2048,
                   steps_min: int = 1000, steps_max: int = 20000):
    """Config 5 request stream (without arrival times): lattice side s
    log-uniform in [side_min, side_max] (rounded to a multiple of 16), steps
    uniform in [steps_min, steps_max], kind uniform over the three single-lattice
    cases:

      cavity    s x s lid-driven cavity, BGK tau 0.884, lid u = (0.1, 0)
      cylinder  (s/4) x s channel (at least 32 rows), TRT magic 1/4, parabolic
                Zou-He inlet u_max 0.05, Zou-He pressure outlet rho 1, staircase
                cylinder of radius 20/256 of the height at (200/1024, 131/256)
                of the channel, tau from Re 200: nu = 0.05 * 2r / 200
      porous    s x s random porous channel (discs r 3..12, 30 % solid, seed
                from the side), BGK tau 0.8, Zou-He inlet u 0.02, Zou-He
                pressure outlet rho 1

    numpy PCG64 with a fixed seed.  Each request is a dict with `make_types()`
    and `open_values(lists)` (one row of boundary values, repeated for every
    step)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for q in range(n):
        side = int(round(np.exp(rng.uniform(np.log(side_min), np.log(side_max))) / 16.0)) * 16
        side = min(max(side, side_min), side_max)
        steps = int(rng.integers(steps_min, steps_max + 1))
        kind = ("cavity", "cylinder", "porous")[int(rng.integers(0, 3))]
        if kind == "cavity":
            R, C = side, side
            req = dict(collision=0, tau=0.884, tau_even=0.884, tau_odd=0.884, outlet_bc=0)
            make = (lambda s=side: cavity_types(s))
            lid = 0.1
        elif kind == "cylinder":
            R, C = max(32, side // 4), side
            r = max(3, int(round(20.0 * R / 256.0)))
            tau = 3.0 * (0.05 * 2 * r / 200.0) + 0.5
            req = dict(collision=1, tau=tau, tau_even=tau, tau_odd=0.25 / (tau - 0.5) + 0.5, outlet_bc=2)
            x0, y0 = int(round(200.0 * C / 1024.0)), int(round(131.0 * R / 256.0))
            make = (lambda R=R, C=C, x0=x0, y0=y0, r=r: cylinder_types(R, C, x0, y0, r))
            lid = None
        else:
            R, C = side, side
            req = dict(collision=0, tau=0.8, tau_even=0.8, tau_odd=0.8, outlet_bc=2)
            make = (lambda s=side: porous_types(s, s, seed=20261203 + s))
            lid = None
        req.update(kind=kind, rows=R, cols=C, steps=steps, make_types=make, lid=lid)
        out.append(req)
    return out


def serve_open_values(req: dict, lists: dict) -> np.ndarray:
    """One row of boundary values for a config-5 request (inlets, then outlets)."""
    ni, no = len(lists["inlet"]), len(lists["outlet"])
    t = np.zeros((1, ni + no, 2))
    if req["kind"] == "cavity":
        t[0, :ni, 0] = req["lid"]
    elif req["kind"] == "cylinder":
        R = req["rows"]
        for q, (i, _) in enumerate(lists["inlet"]):
            t[0, q, 0] = parabolic_u(int(i), 0.05, 1, R - 2)
        t[0, ni:] = (1.0, 0.0)
    else:
        t[0, :ni, 0] = 0.02
        t[0, ni:] = (1.0, 0.0)
    return t


def poisson_arrivals(n: int, rate_per_s: float, seed: int = 20261206) -> np.ndarray:
    """Arrival times (seconds from 0) of a Poisson process: exponential gaps."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.cumsum(rng.exponential(1.0 / rate_per_s, size=n))
