"""Synthetic problems: the reference's generators and the project-defined workloads.

All randomness comes from a portable splitmix64 stream (uniform = (u >> 11) * 2^-53), so
the same seed gives the same matrix and right-hand side on every machine.

- poisson_2d(n)                     SparseMatrix::poisson_2d (sparse_matrix.cpp:288-311)
- convection_diffusion_2d(n, ...)   SparseMatrix::convection_diffusion_2d (:317-350)
- varkappa_poisson_2d(n, sigma, s)  -div(kappa grad u) = f, 5-point, lognormal kappa per
                                    cell, harmonic face averages; no reference counterpart
- helmholtz_2d(n, c)                poisson_2d with c added on the diagonal
CSR arrays come back as (row_ptr int32, col_idx int32, values float64) with sorted
columns, i.e. what the reference's from_coo produces.
"""
from __future__ import annotations

import math

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, count: int, offset: int = 0) -> np.ndarray:
    """`count` outputs of the splitmix64 generator started at `seed`, skipping `offset`."""
    with np.errstate(over="ignore"):
        k = np.arange(offset + 1, offset + count + 1, dtype=np.uint64)
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + k * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return z


def uniform(seed: int, count: int, lo: float = 0.0, hi: float = 1.0, offset: int = 0) -> np.ndarray:
    u = (splitmix64(seed, count, offset) >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)
    if lo == 0.0 and hi == 1.0:
        return u
    return lo + (hi - lo) * u


def normal(seed: int, count: int, offset: int = 0) -> np.ndarray:
    """Box-Muller on pairs of the uniform stream."""
    u = uniform(seed, 2 * count, offset=2 * offset)
    u1, u2 = u[0::2], u[1::2]
    return np.sqrt(-2.0 * np.log1p(-u1)) * np.cos(2.0 * math.pi * u2)


def _assemble_5pt(n: int, north, west, diag, east, south):
    """CSR of a 5-point operator on an n x n grid in natural order; the off-diagonal
    arrays hold values per node and are ignored where the neighbour is off the grid."""
    N = n * n
    ii, jj = np.divmod(np.arange(N, dtype=np.int64), n)
    has = [ii > 0, jj > 0, np.ones(N, bool), jj < n - 1, ii < n - 1]
    offs = [-n, -1, 0, 1, n]
    vals = [north, west, diag, east, south]
    counts = sum(h.astype(np.int32) for h in has)
    rp = np.zeros(N + 1, dtype=np.int32)
    np.cumsum(counts, out=rp[1:])
    nnz = int(rp[-1])
    ci = np.empty(nnz, dtype=np.int32)
    v = np.empty(nnz, dtype=np.float64)
    slot = rp[:-1].astype(np.int64).copy()
    node = np.arange(N, dtype=np.int64)
    for h, o, val in zip(has, offs, vals):
        idx = slot[h]
        ci[idx] = (node[h] + o).astype(np.int32)
        v[idx] = val[h] if isinstance(val, np.ndarray) else val
        slot[h] += 1
    return rp, ci, v


def poisson_2d(n: int):
    N = n * n
    return _assemble_5pt(n, -1.0, -1.0, np.full(N, 4.0), -1.0, -1.0)


def convection_diffusion_2d(n: int, eps: float = 1.0, bx: float = 0.0, by: float = 0.0):
    """Same arithmetic, in the same order, as sparse_matrix.cpp:317-350."""
    N = n * n
    h = 1.0 / (n + 1)
    eh = eps / (h * h)
    bxh = bx / (2.0 * h)
    byh = by / (2.0 * h)
    ii, jj = np.divmod(np.arange(N, dtype=np.int64), n)
    diag = np.full(N, 4.0 * eh)
    diag = np.where(jj > 0, diag + max(-bxh, 0.0), diag)
    diag = np.where(jj < n - 1, diag + max(bxh, 0.0), diag)
    diag = np.where(ii > 0, diag + max(-byh, 0.0), diag)
    diag = np.where(ii < n - 1, diag + max(byh, 0.0), diag)
    west = -eh + max(bxh, 0.0)
    east = -eh - min(bxh, 0.0)
    north = -eh + max(byh, 0.0)
    south = -eh - min(byh, 0.0)
    return _assemble_5pt(n, north, west, diag, east, south)


def convdiff_wind(n: int, peclet: float, eps: float = 1.0, angle_deg: float = 30.0):
    """(bx, by) for cell Peclet number Pe = |w| h / (2 eps), h = 1/(n+1)."""
    w = 2.0 * peclet * eps * (n + 1)
    a = math.radians(angle_deg)
    return w * math.cos(a), w * math.sin(a)


def varkappa_poisson_2d(n: int, sigma: float = 1.0, seed: int = 0):
    """-div(kappa grad u) with kappa = exp(sigma * N(0,1)) per cell, harmonic face averages
    2 kP kQ / (kP + kQ), boundary faces kP; diag = sum of the four faces, off = -face."""
    N = n * n
    kap = np.exp(sigma * normal(seed, N)).reshape(n, n)
    fx = 2.0 * kap[:, :-1] * kap[:, 1:] / (kap[:, :-1] + kap[:, 1:])   # face (i,j)-(i,j+1)
    fy = 2.0 * kap[:-1, :] * kap[1:, :] / (kap[:-1, :] + kap[1:, :])   # face (i,j)-(i+1,j)
    west = np.empty((n, n)); west[:, 0] = kap[:, 0]; west[:, 1:] = fx
    east = np.empty((n, n)); east[:, -1] = kap[:, -1]; east[:, :-1] = fx
    north = np.empty((n, n)); north[0, :] = kap[0, :]; north[1:, :] = fy
    south = np.empty((n, n)); south[-1, :] = kap[-1, :]; south[:-1, :] = fy
    diag = ((north + west) + east) + south
    return _assemble_5pt(n, -north.ravel(), -west.ravel(), diag.ravel(), -east.ravel(),
                         -south.ravel())


def helmholtz_2d(n: int, c: float):
    rp, ci, v = poisson_2d(n)
    rows = np.repeat(np.arange(n * n), np.diff(rp))
    v[ci == rows] += c
    return rp, ci, v


def rhs(n_rows: int, seed: int, lo: float = 0.0, hi: float = 1.0) -> np.ndarray:
    return uniform(seed, n_rows, lo, hi, offset=1 << 40)


def serving_specs(count: int, seed: int, n_lo: float = 1e3, n_hi: float = 4.2e6,
                  rate: float = 0.0):
    """The requests of serving_stream(...) as specs (kind, side, parameter, seed, arrival_s),
    without building them: build_request(spec) makes (rp, ci, v, b, arrival_s, kind) when it
    is needed, so long streams of large systems need not be held in memory at once."""
    u = uniform(seed, 6 * count).reshape(count, 6)
    t = 0.0
    out = []
    for k in range(count):
        n = math.exp(math.log(n_lo) + u[k, 0] * (math.log(n_hi) - math.log(n_lo)))
        side = max(8, int(round(math.sqrt(n))))
        rseed = seed * 1_000_003 + k
        if u[k, 1] < 0.5:
            spec = ("varkappa", side, 1.5 * u[k, 2], rseed)
        elif u[k, 1] < 0.85:
            spec = ("convdiff", side, math.exp(u[k, 3] * math.log(1000.0)), rseed)
        else:
            spec = ("helmholtz", side, 0.1 + 9.9 * u[k, 4], rseed)
        if rate > 0:
            t += -math.log1p(-u[k, 5]) / rate
        out.append(spec + (t,))
    return out


def build_request(spec):
    """(rp, ci, v, b, arrival_s, kind) of a serving_specs entry."""
    kind, side, par, rseed, t = spec
    if kind == "varkappa":
        A = varkappa_poisson_2d(side, par, rseed)
    elif kind == "convdiff":
        A = convection_diffusion_2d(side, 1.0, *convdiff_wind(side, par))
    else:
        A = helmholtz_2d(side, par)
    return (*A, rhs(side * side, rseed), t, kind)


def serving_stream(count: int, seed: int, n_lo: float = 1e3, n_hi: float = 4.2e6,
                   rate: float = 0.0):
    """A serving workload: `count` requests (rp, ci, v, b, arrival_s, kind).

    Sizes are log-uniform in [n_lo, n_hi] on square grids (side = round(sqrt(n))).  The mix
    is 50% variable-kappa Poisson (sigma uniform in [0, 1.5]), 35% upwind
    convection-diffusion (cell Peclet log-uniform in [1, 1000]) and 15% shifted Helmholtz
    (c uniform in [0.1, 10]); rhs uniform [0, 1).  Arrivals form a Poisson process of
    `rate` requests/s (exponential gaps); rate 0 puts every arrival at t = 0."""
    return [build_request(sp) for sp in serving_specs(count, seed, n_lo, n_hi, rate)]
