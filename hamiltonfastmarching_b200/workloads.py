"""Seeded synthetic inputs for the solve path, in the reference's ``hfmIn`` key vocabulary.

Every generator returns a plain ``dict`` of numpy float64 arrays / scalars / strings that can be
handed unchanged to the reference's FileHFM executables (``arrayOrdering='RowMajor'``, arrays
indexed ``[i, j(, k)]`` along x, y(, z|theta)) or to :class:`hamiltonfastmarching_b200.HFMIO`.

Conventions (shared by the tests, the benchmark and the golden-vector script):

* grid points sit at cell centres ``x_i = origin + (i + 1/2) h`` (reference ``BaseGrid.h:69-75``);
* a *smooth field* is ``K**-0.5 * sum_k A_k cos(2 pi k.x + phi_k)`` over ``K`` random integer
  wave vectors with ``|k|_inf <= 4``, ``A_k ~ N(0,1)``, ``phi_k ~ U[0, 2 pi)``;
* symmetric matrices are packed in the reference's order ``(xx, xy, yy[, xz, yz, zz])``
  (``SymmetricMatrixType.hxx:11-16``), component axis last.

No public dataset is involved; these stand in for the workloads the benchmarks are quoted on.
"""
from __future__ import annotations

import math
from typing import Dict, Tuple

import numpy as np

__all__ = [
    "smooth_field",
    "riemann2_case",
    "riemann3_case",
    "tubular_image",
    "curvature2_case",
    "pack_sym2",
    "pack_sym3",
]


def _grid_axes(shape, h, origin=None):
    origin = np.zeros(len(shape)) if origin is None else np.asarray(origin, float)
    return [origin[d] + (np.arange(n) + 0.5) * h for d, n in enumerate(shape)]


def smooth_field(rng: np.random.Generator, shape, h, K: int = 8, kmax: int = 4,
                 dtype=np.float64) -> np.ndarray:
    """Sum of ``K`` random-phase Fourier modes on the unit-periodic domain, normalised by sqrt(K)."""
    axes = _grid_axes(shape, h)
    d = len(shape)
    out = np.zeros(shape, dtype=dtype)
    for _ in range(K):
        k = rng.integers(-kmax, kmax + 1, size=d)
        amp = rng.standard_normal()
        phase = rng.uniform(0.0, 2.0 * math.pi)
        # cos(A + B) = cos A cos B - sin A sin B, A = phase + ramp of the first axis, B = the
        # ramps of the other axes summed on their (lower-dimensional) grid
        A = phase + 2.0 * math.pi * k[0] * axes[0]
        if d == 1:
            out += amp * np.cos(A).astype(dtype)
            continue
        B = np.zeros(shape[1:])
        for ax in range(1, d):
            sh = [1] * (d - 1)
            sh[ax - 1] = shape[ax]
            B = B + (2.0 * math.pi * k[ax] * axes[ax]).reshape(sh)
        sh0 = (shape[0],) + (1,) * (d - 1)
        cb, sb = np.cos(B)[None], np.sin(B)[None]
        out += (amp * np.cos(A)).reshape(sh0).astype(dtype) * cb - (amp * np.sin(A)).reshape(sh0).astype(dtype) * sb
    out /= math.sqrt(K)
    return out


def pack_sym2(m00, m01, m11) -> np.ndarray:
    return np.stack([m00, m01, m11], axis=-1)


def pack_sym3(m00, m01, m11, m02, m12, m22) -> np.ndarray:
    return np.stack([m00, m01, m11, m02, m12, m22], axis=-1)


def riemann2_case(n: int = 256, aniso: float = 5.0, seed: int = 0, n_seeds: int = 1,
                  seed_points=None) -> Dict:
    """Riemann2 on [0,1]^2, M = R(theta) diag(1, 1/a^2) R(theta)^T with smooth random theta.

    Default arguments reproduce the 256x256, a=5, single centre seed workload.
    """
    rng = np.random.default_rng(seed)
    h = 1.0 / n
    theta = math.pi * smooth_field(rng, (n, n), h)
    c, s = np.cos(theta), np.sin(theta)
    l0, l1 = 1.0, 1.0 / aniso ** 2
    m00 = l0 * c * c + l1 * s * s
    m01 = (l0 - l1) * c * s
    m11 = l0 * s * s + l1 * c * c
    if seed_points is None:
        if n_seeds == 1:
            seed_points = np.array([[0.5, 0.5]])
        else:
            seed_points = rng.uniform(0.05, 0.95, size=(n_seeds, 2))
    return {
        "model": "Riemann2",
        "arrayOrdering": "RowMajor",
        "dims": np.array([n, n], dtype=float),
        "gridScale": h,
        "metric": pack_sym2(m00, m01, m11),
        "seeds": np.asarray(seed_points, dtype=float),
        "exportValues": 1.0,
    }


def _rodrigues(wx, wy, wz):
    """Rotation matrices exp(skew(w)) for fields of axis-angle vectors (returns 3x3 nested lists)."""
    th = np.sqrt(wx * wx + wy * wy + wz * wz)
    small = th < 1e-12
    ths = np.where(small, 1.0, th)
    kx, ky, kz = wx / ths, wy / ths, wz / ths
    c, s = np.cos(th), np.sin(th)
    v = 1.0 - c
    R = [[c + kx * kx * v, kx * ky * v - kz * s, kx * kz * v + ky * s],
         [ky * kx * v + kz * s, c + ky * ky * v, ky * kz * v - kx * s],
         [kz * kx * v - ky * s, kz * ky * v + kx * s, c + kz * kz * v]]
    one = np.ones_like(th)
    zero = np.zeros_like(th)
    eye = [[one, zero, zero], [zero, one, zero], [zero, zero, one]]
    return [[np.where(small, eye[i][j], R[i][j]) for j in range(3)] for i in range(3)]


def riemann3_case(n: int = 192, seed: int = 1, n_spheres: int = 40, n_seeds: int = 16,
                  rmin: float = 0.02, rmax: float = 0.08, walls: bool = True) -> Dict:
    """Riemann3 on [0,1]^3 with M = R diag(1, a1^-2, a2^-2) R^T, spherical walls and random seeds.

    a1, a2 = exp(ln 20 * (1/2 + 1/2 tanh(smooth))) lie in [1, 20]; R = exp(skew(pi * smooth^3)).
    Walls are the union of ``n_spheres`` balls (centres U[0,1]^3, radii U[rmin, rmax]);
    seeds are uniform points whose cell is not a wall.
    """
    rng = np.random.default_rng(seed)
    h = 1.0 / n
    shape = (n, n, n)
    f = lambda: smooth_field(rng, shape, h)
    a1 = np.exp(math.log(20.0) * (0.5 + 0.5 * np.tanh(f())))
    a2 = np.exp(math.log(20.0) * (0.5 + 0.5 * np.tanh(f())))
    w = [math.pi * f() for _ in range(3)]
    R = _rodrigues(*w)
    lam = [np.ones(shape), a1 ** -2, a2 ** -2]
    del a1, a2, w

    def m(i, j):
        return sum(R[i][k] * lam[k] * R[j][k] for k in range(3))

    metric = pack_sym3(m(0, 0), m(0, 1), m(1, 1), m(0, 2), m(1, 2), m(2, 2))
    del R, lam
    out = {
        "model": "Riemann3",
        "arrayOrdering": "RowMajor",
        "dims": np.array([n, n, n], dtype=float),
        "gridScale": h,
        "metric": metric,
        "exportValues": 1.0,
    }
    wall = np.zeros(shape, dtype=bool)
    if walls and n_spheres > 0:
        ax = _grid_axes(shape, h)
        centres = rng.uniform(0.0, 1.0, size=(n_spheres, 3))
        radii = rng.uniform(rmin, rmax, size=n_spheres)
        for c, r in zip(centres, radii):
            lo = np.clip(np.floor((c - r) / h).astype(int) - 1, 0, n)
            hi = np.clip(np.ceil((c + r) / h).astype(int) + 1, 0, n)
            X = ax[0][lo[0]:hi[0]].reshape(-1, 1, 1)
            Y = ax[1][lo[1]:hi[1]].reshape(1, -1, 1)
            Z = ax[2][lo[2]:hi[2]].reshape(1, 1, -1)
            inside = (X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2 <= r * r
            wall[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] |= inside
        out["walls"] = wall.astype(float)
    seeds = []
    while len(seeds) < n_seeds:
        p = rng.uniform(0.0, 1.0, size=3)
        idx = np.minimum((p / h).astype(int), n - 1)
        if not wall[tuple(idx)]:
            seeds.append(p)
    out["seeds"] = np.array(seeds, dtype=float)
    return out


def tubular_image(rng: np.random.Generator, n: int, n_curves: int = 20, width_px: float = 2.0,
                  samples: int = 400) -> np.ndarray:
    """Max over random cubic Bezier curves of the Gaussian profile exp(-d^2 / (2 (width h)^2))."""
    h = 1.0 / n
    ax = (np.arange(n) + 0.5) * h
    X, Y = np.meshgrid(ax, ax, indexing="ij")
    img = np.zeros((n, n))
    sig = width_px * h
    t = np.linspace(0.0, 1.0, samples)
    b = np.stack([(1 - t) ** 3, 3 * t * (1 - t) ** 2, 3 * t ** 2 * (1 - t), t ** 3], axis=1)
    for _ in range(n_curves):
        P = rng.uniform(0.0, 1.0, size=(4, 2))
        curve = b @ P  # (samples, 2)
        d2 = np.full((n, n), np.inf)
        # distance to the sampled polyline, evaluated on a bounding window only
        lo = np.clip(((curve.min(0) - 4 * sig) / h).astype(int), 0, n)
        hi = np.clip(((curve.max(0) + 4 * sig) / h).astype(int) + 1, 0, n)
        Xw = X[lo[0]:hi[0], lo[1]:hi[1]]
        Yw = Y[lo[0]:hi[0], lo[1]:hi[1]]
        dw = np.full(Xw.shape, np.inf)
        for q in curve:
            np.minimum(dw, (Xw - q[0]) ** 2 + (Yw - q[1]) ** 2, out=dw)
        d2[lo[0]:hi[0], lo[1]:hi[1]] = dw
        np.maximum(img, np.exp(-d2 / (2.0 * sig * sig)), out=img)
    return img


def curvature2_case(n: int = 128, ntheta: int = 60, model: str = "ReedsShepp2", seed: int = 2,
                    xi: float = 0.1, eps: float = 0.1, n_curves: int = 20, n_seeds: int = 1,
                    seed_points=None) -> Dict:
    """ReedsShepp2 / Elastica2 on the lifted grid (x, y, theta) of n x n x ntheta points.

    The cost is the physical (n, n) field 1/(0.05 + I) with I a synthetic tubular image;
    seeds are full (x, y, theta) points.
    """
    rng = np.random.default_rng(seed)
    img = tubular_image(rng, n, n_curves=n_curves)
    cost = 1.0 / (0.05 + img)
    if seed_points is None:
        pts = rng.uniform(0.2, 0.8, size=(n_seeds, 2))
        th = rng.uniform(0.0, 2.0 * math.pi, size=(n_seeds, 1))
        seed_points = np.concatenate([pts, th], axis=1)
    return {
        "model": model,
        "arrayOrdering": "RowMajor",
        "dims": np.array([n, n, ntheta], dtype=float),
        "gridScale": 1.0 / n,
        "xi": float(xi),
        "eps": float(eps),
        "cost": cost,
        "seeds": np.asarray(seed_points, dtype=float),
        "exportValues": 1.0,
    }


def reedsshepp3_case(n: int = 32, ntheta: int = 8, seed: int = 6, xi: float = 0.3, eps: float = 0.1,
                     dual: bool = False, projective: bool = False, cost: str = "spatial", n_seeds: int = 1) -> Dict:
    """ReedsShepp3 on the grid (x, y, z, theta, phi) of n^3 x ntheta x nphi points, nphi = 2 ntheta
    (4 ntheta projective). The cost is 1 + |smooth field| over (x, y, z) ("spatial"), over
    (theta, phi) ("angular"), over the whole grid ("full"), or 1.5 ("constant"); seeds are full
    5-D points."""
    rng = np.random.default_rng(seed)
    nphi = (4 if projective else 2) * ntheta
    dims = (n, n, n, ntheta, nphi)
    if cost == "spatial":
        c = 1.0 + np.abs(smooth_field(rng, (n, n, n), 1.0 / n))
    elif cost == "angular":
        c = 1.0 + np.abs(smooth_field(rng, (ntheta, nphi), 1.0 / nphi))
    elif cost == "full":
        c = 1.0 + np.abs(smooth_field(rng, dims, 1.0 / n))
    else:
        c = 1.5
    pts = rng.uniform(0.3, 0.7, size=(n_seeds, 3))
    theta = rng.uniform(0.1, (0.5 if projective else 1.0) * math.pi - 0.1, size=(n_seeds, 1))
    phi = rng.uniform(0.0, 2.0 * math.pi, size=(n_seeds, 1))
    return {
        "model": "ReedsShepp3",
        "arrayOrdering": "RowMajor",
        "dims": np.array(dims, dtype=float),
        "gridScale": 1.0 / n,
        "xi": float(xi),
        "eps": float(eps),
        "dual": float(bool(dual)),
        "projective": float(bool(projective)),
        "cost": c,
        "seeds": np.concatenate([pts, theta, phi], axis=1),
        "exportValues": 1.0,
    }


def thomsen_tti(vp, eps, delta, dip, azimuth) -> np.ndarray:
    """TTI metric elements (..., 14) from Thomsen parameters and tilt angles.

    The qP slowness surface is taken in Alkhalifah's acoustic approximation of transversely
    isotropic media (Geophysics 63(2), 1998; 65(4), 2000): with p_h, p_v the slowness components
    across and along the symmetry axis,
        vh^2 p_h^2 + vv^2 p_v^2 - 2 eta vn^2 vv^2 p_h^2 p_v^2 = 1,
    vv = vp, vh^2 = vp^2 (1 + 2 eps), vn^2 = vp^2 (1 + 2 delta), eta = (eps - delta) / (1 + 2 delta).
    That is the reference's algebraic form <linear, q> + 1/2 <q, quadratic, q> = 1 with
    q = (p_h^2, p_v^2): linear = (vh^2, vv^2), quadratic = (0, -2 vp^4 (eps - delta), 0). The
    transform is the rotation whose last row is the symmetry axis (dip from the vertical, then
    azimuth), so that its rows give (p_h components, p_v) of a slowness vector.
    """
    vp, eps, delta, dip, azimuth = np.broadcast_arrays(*(np.asarray(a, float) for a in (vp, eps, delta, dip, azimuth)))
    out = np.zeros(vp.shape + (14,))
    vp2 = vp * vp
    out[..., 0] = vp2 * (1 + 2 * eps)
    out[..., 1] = vp2
    out[..., 2] = 0.0
    out[..., 3] = -2.0 * vp2 * vp2 * (eps - delta)
    out[..., 4] = 0.0
    sd, cd, sa, ca = np.sin(dip), np.cos(dip), np.sin(azimuth), np.cos(azimuth)
    # rows: e1 = (cd ca, cd sa, -sd), e2 = (-sa, ca, 0), n = (sd ca, sd sa, cd)
    rows = [(cd * ca, cd * sa, -sd), (-sa, ca, 0 * sd), (sd * ca, sd * sa, cd)]
    # element 5 + i + 3 j holds rows[i][j]; the reference reads the transform row by row, so its
    # transform is this rotation transposed, whose inverse transpose (the map its dual unit ball
    # applies to a slowness vector) is this rotation again
    for i in range(3):
        for j in range(3):
            out[..., 5 + i + 3 * j] = rows[i][j]
    return out


def tti3_case(n: int = 128, h: float = 0.01, seed: int = 4, vp_scale: float = 1.0, blob=None) -> Dict:
    """TTI3 on an n^3 grid of spacing h (km): vp = 1.5 + 3 (1/2 + 1/2 tanh(smooth)) km/s,
    Thomsen eps, delta in [0, 0.2] (delta <= eps) from smooth fields, tilt dip <= 30 degrees and
    uniform azimuth from smooth fields; one source at the centre of the top face (z = 0).
    ``blob`` = (centre (3,), radius, amplitude) multiplies vp by 1 + amplitude exp(-|x-c|^2/(2 r^2)).
    """
    rng = np.random.default_rng(seed)
    shape = (n, n, n)
    L = n * h
    f = lambda: smooth_field(rng, shape, 1.0 / n)
    vp = 1.5 + 3.0 * (0.5 + 0.5 * np.tanh(f()))
    e = 0.2 * (0.5 + 0.5 * np.tanh(f()))
    d = e * (0.5 + 0.5 * np.tanh(f()))
    dip = (math.pi / 6) * (0.5 + 0.5 * np.tanh(f()))
    az = math.pi * (1.0 + np.tanh(f()))
    if blob is not None:
        c, r, amp = blob
        ax = _grid_axes(shape, h)
        X, Y, Z = np.meshgrid(*ax, indexing="ij")
        vp = vp * (1.0 + amp * np.exp(-((X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2) / (2 * r * r)))
    vp = vp * vp_scale
    return {
        "model": "TTI3",
        "arrayOrdering": "RowMajor",
        "dims": np.array([n, n, n], dtype=float),
        "gridScale": h,
        "metric": thomsen_tti(vp, e, d, dip, az),
        "seeds": np.array([[L / 2, L / 2, h / 2]]),
        "exportValues": 1.0,
        "_vp": vp,
    }


def _make(spec):
    fn, kwargs = spec
    return globals()[fn](**kwargs)


def generate(specs, processes: int = 0) -> list:
    """Builds the cases of a list of (generator name, keyword arguments) specs, in a pool of
    ``processes`` worker processes (spawned, so it is safe after CUDA initialisation) when > 1."""
    if processes and processes > 1 and len(specs) > 1:
        import multiprocessing as mp
        with mp.get_context("spawn").Pool(min(processes, len(specs))) as pool:
            return pool.map(_make, specs, chunksize=1)
    return [_make(sp) for sp in specs]


def batched_mix_specs(n_riemann: int = 384, n_lifted: int = 128, ntheta: int = 60, seed: int = 3,
                      side_range=(64, 1024), lifted_range=(64, 256)) -> list:
    """Specs of the mixed batch: Riemann2 instances with log-uniform sides, anisotropy U[1,10] and
    smooth random theta, plus ReedsShepp2 / Elastica2 lifted grids (half each) of N x N x ntheta
    points with the tubular-image cost 1/(0.05+I), xi = 0.1, eps = 0.1. One seed per instance
    (centre for Riemann2, a random oriented point for the lifted models), in a seeded random order.
    """
    rng = np.random.default_rng(seed)
    lo, hi = np.log(side_range[0]), np.log(side_range[1])
    sides = np.exp(rng.uniform(lo, hi, n_riemann)).round().astype(int)
    anisos = rng.uniform(1.0, 10.0, n_riemann)
    llo, lhi = np.log(lifted_range[0]), np.log(lifted_range[1])
    lsides = np.exp(rng.uniform(llo, lhi, n_lifted)).round().astype(int)
    specs = []
    for k in range(n_riemann):
        specs.append(("riemann2_case", dict(n=int(sides[k]), aniso=float(anisos[k]), seed=int(seed * 100003 + k))))
    for k in range(n_lifted):
        model = "ReedsShepp2" if k % 2 == 0 else "Elastica2"
        specs.append(("curvature2_case", dict(n=int(lsides[k]), ntheta=ntheta, model=model,
                                              seed=int(seed * 100003 + n_riemann + k), xi=0.1, eps=0.1)))
    order = rng.permutation(len(specs))
    return [specs[i] for i in order]


def batched_mix(n_riemann: int = 384, n_lifted: int = 128, ntheta: int = 60, seed: int = 3,
                side_range=(64, 1024), lifted_range=(64, 256), precision: str = "float32",
                processes: int = 0) -> list:
    """The mixed batch of ``batched_mix_specs`` as a list of hfmIn dictionaries."""
    cases = generate(batched_mix_specs(n_riemann, n_lifted, ntheta, seed, side_range, lifted_range), processes)
    for p in cases:
        p["solverPrecision"] = precision
    return cases


def serving_specs(n_requests: int, seed: int = 5, ntheta: int = 60) -> list:
    """Specs of a serving request mix: 60% Riemann2 (sides log-uniform 64-1024), 25% Riemann3
    (sides 64-192, 40 spherical walls), 15% ReedsShepp2 (N x N x ntheta, N 64-256, tubular-image
    cost, xi = 0.1); 1-4 random seeds each; every request has its own field seed."""
    rng = np.random.default_rng(seed)
    specs = []
    for k in range(n_requests):
        u = rng.uniform()
        ns = int(rng.integers(1, 5))
        fs = int(seed * 1000003 + k)
        if u < 0.60:
            n = int(round(np.exp(rng.uniform(np.log(64), np.log(1024)))))
            specs.append(("riemann2_case", dict(n=n, aniso=float(rng.uniform(1, 10)), seed=fs, n_seeds=ns)))
        elif u < 0.85:
            n = int(round(np.exp(rng.uniform(np.log(64), np.log(192)))))
            specs.append(("riemann3_case", dict(n=n, seed=fs, n_seeds=ns)))
        else:
            n = int(round(np.exp(rng.uniform(np.log(64), np.log(256)))))
            specs.append(("curvature2_case", dict(n=n, ntheta=ntheta, model="ReedsShepp2", seed=fs, xi=0.1,
                                                  n_seeds=ns)))
    return specs
