"""Synthetic input sets with the shapes of the reference preprocessor's output.

The reference preprocessor (preprocessor/main.cpp) hard-codes R=125 mm,
dx=0.5 mm, m=4 and an amplitude-1 pulse.  This module builds the same kind of
file set for any R, dx, m, nu and pulse:

* the node lattice exactly as preprocessor/main.cpp:851-858 builds it
  (accumulated ``x += dx`` loops, x outer, y inner, r <= R + 1e-10);
* the absorbing ring r > R - delta (:867-873) with every ring node active;
* clouds: all nodes within delta + 1e-10 of each ring node, in node order
  (:884-902), padded with -1 to maxCloudSize;
* the initial displacement either as the reference preprocessor writes it
  (``pulse="reference"``: u_x = u_y = exp(-r^2/100) for r < 40, :1280-1289)
  or as a radial Gaussian u = A exp(-(|x-c|/sigma)^2) (x-c)/|x-c|; v = 0.

Absorbing-boundary operators:

* ``abc="lsq"`` -- the reference preprocessor's own: the least-squares
  plane-wave fit of G_u, G_v and G_theta (:415-785) and, unless ``dt`` is
  given, the (dt, delta_kappa) stability sweep that picks the time step
  (:1047-1174), computed by ``abcfit`` (the host C++ fit in liblps_b200.so);
* ``abc="average"`` -- passive operators of the same shapes and density whose
  rows average the cloud's current level (weights 1/C_i on x->x, y->y and
  theta^n, zero on the n-1 level); runs stay bounded, but nothing is absorbed;
* ``abc="none"`` -- no absorbing layer (constrainsNo = 0).
"""
from __future__ import annotations

import math

import numpy as np

from .files import InputSet

STEEL_E = 190.0 / 1000.0        # preprocessor/main.cpp:58
STEEL_RHO = 8000.0 / 1e18       # :60
STEEL_G0 = 22170.0 * 1e-9       # :61


def disc_lattice(R: float, dx: float, dy: float | None = None) -> np.ndarray:
    """Nodes of the disc r <= R on the dx lattice, in the preprocessor's order."""
    dy = dx if dy is None else dy
    xs = []
    x = -R
    while x <= R + 1e-10:
        xs.append(x)
        x += dx
    ys = []
    y = -R
    while y <= R + 1e-10:
        ys.append(y)
        y += dy
    X, Y = np.meshgrid(np.array(xs), np.array(ys), indexing="ij")
    keep = np.sqrt(X * X + Y * Y) <= R + 1e-10
    return np.stack([X[keep], Y[keep]], axis=1)


def lattice_index(nodes: np.ndarray, dx: float, dy: float):
    x0, y0 = nodes[:, 0].min(), nodes[:, 1].min()
    ix = np.rint((nodes[:, 0] - x0) / dx).astype(np.int64)
    iy = np.rint((nodes[:, 1] - y0) / dy).astype(np.int64)
    return ix, iy


def clouds_of(nodes: np.ndarray, centres: np.ndarray, radius: float, dx: float, dy: float):
    """Node indices within `radius` (+1e-10) of each centre node, ascending."""
    ix, iy = lattice_index(nodes, dx, dy)
    nx, ny = ix.max() + 1, iy.max() + 1
    grid = -np.ones((nx, ny), np.int64)
    grid[ix, iy] = np.arange(nodes.shape[0])
    r = int(math.ceil(radius / min(dx, dy))) + 1
    offs = [(a, b) for a in range(-r, r + 1) for b in range(-r, r + 1)]
    cols = []
    for a, b in offs:
        jx, jy = ix[centres] + a, iy[centres] + b
        ok = (jx >= 0) & (jx < nx) & (jy >= 0) & (jy < ny)
        j = np.where(ok, grid[np.clip(jx, 0, nx - 1), np.clip(jy, 0, ny - 1)], -1)
        d = nodes[np.maximum(j, 0)] - nodes[centres]
        dist = np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1])
        cols.append(np.where((j >= 0) & (dist <= radius + 1e-10), j, -1))
    M = np.stack(cols, axis=1)
    M = np.where(M < 0, np.iinfo(np.int64).max, M)
    M.sort(axis=1)
    cnt = (M != np.iinfo(np.int64).max).sum(axis=1)
    C = int(cnt.max()) if cnt.size else 0
    M = M[:, :C]
    M = np.where(M == np.iinfo(np.int64).max, -1, M)
    return M.astype(np.int32), C


def disc_problem(R: float = 125.0, dx: float = 0.5, m: int = 4, nu: float = 0.25,
                 E: float = STEEL_E, rho: float = STEEL_RHO, dt: float | None = None,
                 n_steps: int = 4000, pulse="baseline", amplitude: float = 1e-3,
                 sigma: float | None = None, centre=(0.0, 0.0), abc: str = "average",
                 abcs_step: int = 2, jitter: float = 0.0, seed: int = 0, dk_factor: float = 1.0,
                 fit_threads: int = 0) -> InputSet:
    """Build one input set (see the module docstring).  ``dt``: the time step;
    None means 17.5 ns (the reference preprocessor's pick at nu=0.25) for
    ``abc`` "average" and "none", and the stability sweep's pick for "lsq"
    (given a dt, "lsq" fits at that dt and delta_kappa = dk_factor /
    sqrt(c_P)).  ``jitter`` > 0 moves every node by a seeded uniform offset of
    up to jitter*dx per coordinate, so the node set is no longer a lattice
    (horizons then come from the distance search alone, as for an arbitrary
    node file)."""
    dy = dx
    delta = m * dx
    nodes = disc_lattice(R, dx, dy)
    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        nodes = nodes + rng.uniform(-jitter * dx, jitter * dx, size=nodes.shape)
    N = nodes.shape[0]
    r = np.sqrt(nodes[:, 0] ** 2 + nodes[:, 1] ** 2)
    u0 = np.zeros(2 * N)
    if pulse == "reference":
        val = np.where(r < 40.0, np.exp(-(r * r) / 100.0), 0.0)
        u0[0::2] = val
        u0[1::2] = val
    elif pulse == "baseline":
        sig = (40.0 / 3.0) if sigma is None else sigma
        d = nodes - np.asarray(centre, np.float64)[None, :]
        rr = np.sqrt(d[:, 0] ** 2 + d[:, 1] ** 2)
        g = amplitude * np.exp(-(rr / sig) ** 2)
        with np.errstate(invalid="ignore", divide="ignore"):
            ux = np.where(rr > 0, g * d[:, 0] / rr, 0.0)
            uy = np.where(rr > 0, g * d[:, 1] / rr, 0.0)
        u0[0::2] = ux
        u0[1::2] = uy
    else:
        raise ValueError(f"unknown pulse {pulse!r}")
    v0 = np.zeros(2 * N)
    bct = -np.ones(2 * N, np.int32)
    if dt is None and abc != "lsq":
        dt = 17.5e-9
    s = InputSet(n_nodes=N, n_steps=n_steps, n_abc=0, max_cloud=0, E=E, nu=nu, rho=rho, dt=dt,
                 delta=delta, dx=dx, dy=dy, nodes=nodes, bctypes=bct, u0=u0, v0=v0,
                 t1=n_steps * (dt or 0.0), s0=math.sqrt(5.0 * math.pi * STEEL_G0 / (12.0 * E * delta)))
    if abc == "none":
        return s
    if abc not in ("average", "lsq"):
        raise ValueError(f"unknown abc {abc!r}")
    ring = np.nonzero(r > R - delta)[0].astype(np.int32)
    clouds, C = clouds_of(nodes, ring, delta, dx, dy)
    NA = ring.size
    bct[2 * ring] = 1
    bct[2 * ring + 1] = 1
    s.n_abc, s.max_cloud = NA, C
    s.inf_nodes, s.clouds = ring, clouds
    s.bctypes = bct
    if abc == "lsq":
        from . import abcfit
        f = abcfit.fit(nodes, ring, clouds, E=E, nu=nu, rho=rho, delta=delta, dx=dx, dy=dy, abcs_step=abcs_step,
                       sweep=dt is None, dt=dt, dk_factor=dk_factor, n_threads=fit_threads)
        s.dt = f["dt"]
        s.t1 = n_steps * s.dt
        s.gu, s.gv, s.gtheta = f["gu"], f["gv"], f["gtheta"]
        s.fit = {k: v for k, v in f.items() if k not in ("gu", "gv", "gtheta")}
        return s
    cnt = (clouds >= 0).sum(axis=1).astype(np.float64)
    w = np.where(clouds >= 0, 1.0 / cnt[:, None], 0.0)
    cpc = 2 * abs(abcs_step)
    gu = np.zeros((2 * NA, cpc * C))
    gu[0::2, 0::cpc] = w      # x^{n} -> x
    gu[1::2, 1::cpc] = w      # y^{n} -> y
    gth = np.zeros((NA, abs(abcs_step) * C))
    gth[:, 0::abs(abcs_step)] = w
    s.gu, s.gv, s.gtheta = gu, gu.copy(), gth
    return s


def poisson_batch(nus=(0.15, 0.20, 0.25, 0.30, 0.35, 0.40, 0.45), **kw) -> list[InputSet]:
    """Seven Example-1 geometries that differ in nu (the Poisson-ratio batch)."""
    return [disc_problem(nu=nu, **kw) for nu in nus]
