"""ctypes front-end of the C oracle (``oracle/fm_oracle.c``).

TEST INFRASTRUCTURE ONLY: used by ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s
CPU-baseline leg as the checker; the product path never imports it.

:func:`solve` takes an ``hfmIn``-style dict (RowMajor arrays) and reproduces the reference's
``Run`` for the Eulerian models Riemann2/3, ReedsShepp2, Elastica2 (and Isotropic2 as a
Riemann metric ``cost^2 Id``) with seeds and walls: the input semantics follow
``Headers/Base/Implementation/HFM_ParamDefault.hxx`` (point -> index), ``StaticFactoring.hxx:242-393``
(seeds), ``HFM_StencilShare.hxx:61-71`` (speed = 1/cost), ``WallObstructionTest.h:30-36`` (walls).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from typing import Dict

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle_fm.so")
_lib = None

_P = ctypes.c_void_p


class _Problem(ctypes.Structure):
    _fields_ = [
        ("ndim", ctypes.c_int),
        ("dims", ctypes.c_int64 * 3),
        ("periodic", ctypes.c_int * 3),
        ("nfwd", ctypes.c_int),
        ("nsym", ctypes.c_int),
        ("share", ctypes.c_int),
        ("off", _P),
        ("w", _P),
        ("mult", _P),
        ("walls", _P),
        ("nseeds", ctypes.c_int),
        ("seed_index", _P),
        ("seed_value", _P),
        ("has_stop_at_distance", ctypes.c_int),
        ("stop_at_distance", ctypes.c_double),
        ("n_max_accepted", ctypes.c_int64),
        ("nstop_any", ctypes.c_int),
        ("nstop_all", ctypes.c_int),
        ("nstop_any_u", ctypes.c_int),
        ("nstop_all_u", ctypes.c_int),
        ("stop_any", _P),
        ("stop_all", _P),
        ("stop_any_u", _P),
        ("stop_all_u", _P),
        ("var_dim", ctypes.c_int),
        ("mult_vec", _P),
        ("nmax", ctypes.c_int),
        ("fac_values", _P),
        ("fac_grads", _P),
        ("fac_mask", _P),
        ("fac_lo", ctypes.c_int * 3),
        ("fac_dims", ctypes.c_int * 3),
        ("fac_subdomain", ctypes.c_int),
    ]


def build() -> str:
    """Compile the oracle shared library (``make -C oracle``) if needed; returns its path."""
    src = os.path.join(_HERE, "fm_oracle.c")
    if (not os.path.exists(_LIB_PATH)) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        L.fmo_selling_mat.argtypes = [ctypes.c_int, _P, _P, _P]
        L.fmo_riemann_stencils.argtypes = [ctypes.c_int, ctypes.c_int64, _P, ctypes.c_int, _P, _P, _P]
        L.fmo_voronoi1vec.argtypes = [ctypes.c_int, _P, ctypes.c_double, _P, _P]
        L.fmo_reedsshepp2_table.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_int, _P, _P]
        L.fmo_elastica2_table.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_double, _P, _P]
        L.fmo_reedssheppforward2_table.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                                   ctypes.c_double, _P, _P]
        L.fmo_dubins2_table.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, _P, _P]
        L.fmo_fast_marching.argtypes = [ctypes.POINTER(_Problem), _P, _P, _P]
        L.fmo_fast_marching.restype = ctypes.c_int64
        L.fmo_backward_variation.argtypes = [ctypes.POINTER(_Problem), _P, _P, ctypes.c_int, _P, _P,
                                             _P, ctypes.c_int64, _P, _P]
        L.fmo_backward_variation.restype = ctypes.c_int64
        L.fmo_visibility.argtypes = [ctypes.POINTER(_Problem), ctypes.c_int, _P]
        L.fmo_tti_fast_marching.argtypes = [_P, _P, _P, ctypes.c_int, _P, _P, _P, _P]
        L.fmo_tti_fast_marching.restype = ctypes.c_int64
        L.fmo_tti_fast_marching_stop.argtypes = [_P, _P, _P, ctypes.c_int, _P, _P, _P, _P, ctypes.POINTER(_Problem)]
        L.fmo_tti_fast_marching_stop.restype = ctypes.c_int64
        L.fmo_tti_norm.argtypes = [_P, _P, _P]
        L.fmo_tti_prefix_solve.argtypes = [_P, _P, _P, _P, _P, ctypes.POINTER(_Problem), _P]
        L.fmo_tti_prefix_fixed_point.argtypes = [_P, _P, _P, _P, _P, ctypes.POINTER(_Problem), ctypes.c_int]
        L.fmo_tti_backward_variation.argtypes = [_P, _P, _P, _P, _P, ctypes.c_int, _P, _P, _P, ctypes.c_int64,
                                                 _P, _P]
        L.fmo_tti_backward_variation.restype = ctypes.c_int64
        L.fmo_geodesic_discrete.argtypes = [ctypes.POINTER(_Problem), _P, _P, ctypes.c_int, _P, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_double, ctypes.c_int64, _P, _P, _P]
        L.fmo_geodesic_discrete.restype = ctypes.c_int64
        L.fmo_tti_geodesic_discrete.argtypes = [_P, _P, _P, _P, _P, ctypes.c_int, _P, ctypes.c_double,
                                                ctypes.c_double, ctypes.c_double, ctypes.c_int64, _P, _P, _P]
        L.fmo_tti_geodesic_discrete.restype = ctypes.c_int64
        L.fmo_geodesic_flow.argtypes = [ctypes.POINTER(_Problem), _P, _P, _P, _P, _P]
        L.fmo_forward_variation.argtypes = [ctypes.POINTER(_Problem), _P, _P, ctypes.c_int, _P, _P]
        L.fmo_geodesic_ode.argtypes = [ctypes.POINTER(_Problem), _P, _P, ctypes.c_int, _P, ctypes.c_double,
                                       ctypes.c_double, ctypes.c_int64, _P, _P, _P]
        L.fmo_geodesic_ode.restype = ctypes.c_int64
        L.fmo_tti_geodesic_ode.argtypes = [_P, _P, _P, _P, _P, ctypes.c_int, _P, ctypes.c_int, _P, ctypes.c_double,
                                           ctypes.c_double, ctypes.c_int64, _P, _P, _P]
        L.fmo_tti_geodesic_ode.restype = ctypes.c_int64
        L.fmo_tti_forward_variation.argtypes = [_P, _P, _P, _P, _P, ctypes.c_int, _P, _P]
        L.fmo_tti_geodesic_flow.argtypes = [_P, _P, _P, _P, _P, _P, _P, _P]
        L.fmo_rs3_stencil.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_int, _P, _P]
        L.fmo_rsf3_stencil.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_double, _P, _P]
        L.fmo_s2_fast_marching.argtypes = [_P, ctypes.c_int, ctypes.c_int, _P, _P, _P, ctypes.c_int, _P, _P, _P,
                                           _P, _P]
        L.fmo_s2_fast_marching.restype = ctypes.c_int64
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


# ----------------------------------------------------------------------------------- stencils

def selling(mats: np.ndarray, ndim: int):
    """Selling decomposition of packed SPD matrices ``(..., 3|6)`` -> offsets (..., k, 3) int8, weights."""
    mats = np.ascontiguousarray(mats, dtype=np.float64)
    ns = 3 if ndim == 2 else 6
    nk = 3 if ndim == 2 else 6
    flat = mats.reshape(-1, ns)
    off = np.zeros((flat.shape[0], nk, 3), np.int8)
    w = np.zeros((flat.shape[0], nk), np.float64)
    L = lib()
    for i in range(flat.shape[0]):
        row = np.ascontiguousarray(flat[i])
        if L.fmo_selling_mat(ndim, _ptr(row), _ptr(off[i]), _ptr(w[i])):
            raise ValueError(f"matrix {i} is not positive definite")
    return off.reshape(mats.shape[:-1] + (nk, 3)), w.reshape(mats.shape[:-1] + (nk,))


def riemann_stencils(metric: np.ndarray, h, dual: bool = False):
    ndim = 2 if metric.shape[-1] == 3 else 3
    nk = 3 if ndim == 2 else 6
    metric = np.ascontiguousarray(metric, dtype=np.float64)
    n = int(np.prod(metric.shape[:-1]))
    h = np.ascontiguousarray(np.broadcast_to(np.asarray(h, float), (ndim,)), dtype=np.float64)
    off = np.zeros((n, nk, 3), np.int8)
    w = np.zeros((n, nk), np.float64)
    if lib().fmo_riemann_stencils(ndim, n, _ptr(metric), int(dual), _ptr(h), _ptr(off), _ptr(w)):
        raise ValueError("ObtuseSuperbase error : input must be positive definite")
    return off, w


def curvature2_table(model: str, ntheta: int, h: float, xi: float, eps: float, projective=False):
    L = lib()
    if model == "ReedsShepp2":
        off = np.zeros((ntheta, 4, 3), np.int8)
        w = np.zeros((ntheta, 4), np.float64)
        rc = L.fmo_reedsshepp2_table(ntheta, h, xi, eps, int(projective), _ptr(off), _ptr(w))
    elif model == "ReedsSheppForward2":
        off = np.zeros((ntheta, 4, 3), np.int8)
        w = np.zeros((ntheta, 4), np.float64)
        rc = L.fmo_reedssheppforward2_table(ntheta, h, xi, eps, _ptr(off), _ptr(w))
    elif model == "Dubins2":
        off = np.zeros((ntheta, 12, 3), np.int8)
        w = np.zeros((ntheta, 12), np.float64)
        rc = L.fmo_dubins2_table(ntheta, h, xi, eps, _ptr(off), _ptr(w))
    elif model == "Elastica2":
        off = np.zeros((ntheta, 27, 3), np.int8)
        w = np.zeros((ntheta, 27), np.float64)
        rc = L.fmo_elastica2_table(ntheta, h, xi, eps, _ptr(off), _ptr(w))
    else:
        raise ValueError(model)
    if rc:
        raise ValueError("stencil construction failed")
    return off, w


# ----------------------------------------------------------------------------------- problems

def _get(params, key, default=None):
    return params[key] if key in params else default


def _seed_indices(params, adim, dims, periodic):
    """Seeds -> unique row-major indices in increasing order, first value kept
    (``StaticFactoring.hxx:256-274, 384-390``; std::map insert semantics)."""
    if "seeds" not in params:
        return np.zeros(0, np.int64), np.zeros(0)
    pts = np.atleast_2d(np.asarray(params["seeds"], float))
    vals = np.asarray(_get(params, "seedValues", np.zeros(len(pts))), float).ravel()
    if len(vals) != len(pts):
        raise ValueError("Error : Inconsistent size of seedValues.")
    seen = {}
    for p, v in zip(pts, vals):
        q = adim(p)
        idx = [int(math.floor(c)) for c in q]
        ok = True
        for a, n in enumerate(dims):
            if periodic[a]:
                idx[a] %= n
            elif not (0 <= idx[a] < n):
                ok = False
        if not ok:
            continue
        lin = int(np.ravel_multi_index(tuple(idx), dims))
        seen.setdefault(lin, float(v))
    keys = sorted(seen)
    return np.array(keys, np.int64), np.array([seen[k] for k in keys], float)


class Problem:
    """Owns the arrays referenced by the C problem structure."""

    def __init__(self, params: Dict):
        model = params["model"]
        dims = tuple(int(round(d)) for d in np.asarray(params["dims"]).ravel())
        self.model, self.dims = model, dims
        ndim = len(dims)
        self.ndim = ndim
        periodic = [0, 0, 0]
        mult = None
        if model in ("Isotropic2", "Isotropic3"):
            # one symmetric difference per axis, weight 1/h_i^2 times the squared speed
            # (Headers/Specializations/Isotropic.h:11-59); the table is repeated on every index of
            # the last axis so that the shared-stencil indexing applies
            origin = np.asarray(_get(params, "origin", np.zeros(ndim)), float)
            if "gridScales" in params:
                hs = np.asarray(params["gridScales"], float).ravel()
            else:
                hs = np.full(ndim, float(params["gridScale"]))
            scale = hs
            nfwd, nsym, share = 0, ndim, 1
            ncls = dims[-1]
            off = np.zeros((ncls, ndim, 3), np.int8)
            w = np.zeros((ncls, ndim))
            for i in range(ndim):
                off[:, i, i] = 1
                w[:, i] = 1.0 / (hs[i] * hs[i])
            if "speed" in params:
                sp = np.asarray(params["speed"], float)
            else:
                sp = 1.0 / np.asarray(params["cost"], float)
            mult = np.ascontiguousarray(np.broadcast_to(sp, dims), dtype=np.float64)
            adim = lambda p: (np.asarray(p, float) - origin) / hs
        elif model in ("Diagonal2", "Diagonal3"):
            # one symmetric difference per axis, weight (1/h_i^2) * speed_i^2 per cell
            # (Headers/Specializations/Isotropic.h:61-115, EulerianStencil.h:79-81)
            origin = np.asarray(_get(params, "origin", np.zeros(ndim)), float)
            if "gridScales" in params:
                hs = np.asarray(params["gridScales"], float).ravel()
            else:
                hs = np.full(ndim, float(params["gridScale"]))
            scale = hs
            if "speed" in params:
                sp = np.asarray(params["speed"], float)
            else:
                sp = 1.0 / np.asarray(params["cost"], float)
            sp = np.broadcast_to(sp, dims + (ndim,)).reshape(-1, ndim)
            n = sp.shape[0]
            off = np.zeros((n, ndim, 3), np.int8)
            w = np.zeros((n, ndim))
            for i in range(ndim):
                off[:, i, i] = 1
                w[:, i] = (1.0 / (hs[i] * hs[i])) * (sp[:, i] * sp[:, i])
            nfwd, nsym, share = 0, ndim, 0
            self._mult_vec = np.ascontiguousarray(sp, np.float64)  # per-axis first variations
            adim = lambda p: (np.asarray(p, float) - origin) / hs
        elif model in ("Riemann2", "Riemann3"):
            origin = np.asarray(_get(params, "origin", np.zeros(ndim)), float)
            if "gridScales" in params:
                hs = np.asarray(params["gridScales"], float).ravel()
            else:
                hs = np.full(ndim, float(params["gridScale"]))
            dual = "dualMetric" in params
            metric = np.asarray(params["dualMetric" if dual else "metric"], float)
            ns = 3 if ndim == 2 else 6
            if metric.shape == (ns,):
                metric = np.broadcast_to(metric, dims + (ns,))
            off, w = riemann_stencils(np.ascontiguousarray(metric), hs, dual)
            nfwd, nsym, share = 0, off.shape[1], 0
            scale = hs
            adim = lambda p: (np.asarray(p, float) - origin) / hs
        elif model in ("ReedsShepp2", "ReedsSheppForward2", "Elastica2", "Dubins2"):
            periodic = [0, 0, 1]
            h = float(params["gridScale"])
            xi = float(_get(params, "xi", 1.0))
            eps = float(_get(params, "eps", 0.1))
            projective = bool(_get(params, "projective", 0.0)) if model == "ReedsShepp2" else False
            nth = dims[2]
            ds = (math.pi if projective else 2 * math.pi) / nth
            off, w = curvature2_table(model, nth, h, xi, eps, projective)
            if model == "ReedsShepp2":
                nfwd, nsym = 0, 4
            elif model == "ReedsSheppForward2":
                nfwd, nsym = 3, 1
            elif model == "Dubins2":  # two stencils of 6 forward differences (nmax = 2)
                nfwd, nsym = 12, 0
            else:
                nfwd, nsym = 27, 0
            share = 1
            if "speed" in params:
                sp = np.asarray(params["speed"], float)
            else:
                sp = 1.0 / np.asarray(params["cost"], float)
            if sp.ndim == 0:
                sp = np.full(dims, float(sp))
            elif sp.shape == dims[:2]:
                sp = np.repeat(sp[:, :, None], nth, axis=2)
            elif sp.shape == (nth,):
                sp = np.broadcast_to(sp[None, None, :], dims)
            mult = np.ascontiguousarray(sp, dtype=np.float64)
            o = np.asarray(_get(params, "origin", np.zeros(2)), float)
            origin = np.array([o[0], o[1], -ds / 2.0])
            scale = np.array([h, h, ds])
            adim = lambda p: (np.asarray(p, float) - origin) / scale
        else:
            raise NotImplementedError(model)
        self.off = np.ascontiguousarray(off.reshape(-1, nfwd + nsym, 3), dtype=np.int8)
        self.w = np.ascontiguousarray(w.reshape(-1, nfwd + nsym), dtype=np.float64)
        self.nfwd, self.nsym, self.share = nfwd, nsym, share
        self.mult = mult
        self.periodic = periodic
        walls = None
        if "walls" in params:
            wl = np.asarray(params["walls"], float)
            if wl.shape != dims and ndim == 3 and wl.shape == dims[:2]:
                wl = np.repeat(wl[:, :, None], dims[2], axis=2)
            walls = np.ascontiguousarray(wl != 0, dtype=np.uint8)
        self.walls = walls
        self.seed_index, self.seed_value = _seed_indices(params, adim, dims, periodic)
        self._adim = adim
        self.origin, self.scale = np.asarray(origin, float), np.asarray(scale, float)
        s = _Problem()
        s.ndim = ndim
        for a in range(3):
            s.dims[a] = dims[a] if a < ndim else 1
            s.periodic[a] = periodic[a]
        s.nfwd, s.nsym, s.share = nfwd, nsym, share
        s.nmax = 2 if model == "Dubins2" else 1
        s.off, s.w = _ptr(self.off), _ptr(self.w)
        s.mult = _ptr(self.mult)
        s.walls = _ptr(self.walls)
        s.nseeds = len(self.seed_index)
        s.seed_index, s.seed_value = _ptr(self.seed_index), _ptr(self.seed_value)
        self.var_dim = 1
        if getattr(self, "_mult_vec", None) is not None:
            self.var_dim = ndim
            s.var_dim, s.mult_vec = ndim, _ptr(self._mult_vec)
        # stopping criteria (CommonStoppingCriteria.h:95-147): target points out of range are dropped
        if "stopAtDistance" in params:
            s.has_stop_at_distance, s.stop_at_distance = 1, float(params["stopAtDistance"])
        if "nMaxAccepted" in params:
            s.n_max_accepted = int(params["nMaxAccepted"])
        self._stops = {}
        for key, fld, unoriented in (("stopWhenAnyAccepted", "stop_any", False),
                                     ("stopWhenAllAccepted", "stop_all", False),
                                     ("stopWhenAnyAccepted_Unoriented", "stop_any_u", True),
                                     ("stopWhenAllAccepted_Unoriented", "stop_all_u", True)):
            if key not in params:
                continue
            cells = []
            for q in np.atleast_2d(np.asarray(params[key], float)):
                if unoriented:
                    i = self.index_of_point(np.array([q[0], q[1], 0.0]))
                    if i is not None:
                        idx = np.unravel_index(i, dims)
                        cells.append(idx[0] * dims[1] + idx[1])
                else:
                    i = self.index_of_point(q)
                    if i is not None:
                        cells.append(i)
            arr = np.ascontiguousarray(cells, np.int64)
            self._stops[fld] = arr
            setattr(s, "n" + fld, len(arr))
            setattr(s, fld, _ptr(arr))
        self.struct = s

    def index_of_point(self, p):
        q = self._adim(p)
        idx = [int(math.floor(c)) for c in q]
        for a, n in enumerate(self.dims):
            if self.periodic[a]:
                idx[a] %= n
            elif not (0 <= idx[a] < n):
                return None
        return int(np.ravel_multi_index(tuple(idx), self.dims))


def solve(params: Dict, with_active: bool = True) -> Dict:
    """Fast-marching solve of ``params`` on the CPU. Returns values (dims), activeNeighs (uint64),
    nAccepted, MaxStencilWidth and the :class:`Problem` used."""
    P = Problem(params)
    n = int(np.prod(P.dims))
    values = np.empty(n, np.float64)
    active = np.zeros(n, np.uint64) if with_active else None
    mw = ctypes.c_int(0)
    nacc = lib().fmo_fast_marching(ctypes.byref(P.struct), _ptr(values), _ptr(active), ctypes.byref(mw))
    if nacc < 0:
        raise RuntimeError("oracle fast marching failed")
    return {"values": values.reshape(P.dims), "activeNeighs": active, "nAccepted": int(nacc),
            "MaxStencilWidth": int(mw.value), "problem": P}


def backward_variation(res: Dict, points, weights=None):
    """Reverse first variation from weighted physical points (one ``inspectSensitivity`` group)."""
    P: Problem = res["problem"]
    pts = np.atleast_2d(np.asarray(points, float))
    wts = np.ones(len(pts)) if weights is None else np.asarray(weights, float).ravel()
    idx = []
    for p in pts:
        i = P.index_of_point(p)
        if i is None:
            raise ValueError("Error : inspectSensitivity data points are out of range")
        idx.append(i)
    idx = np.array(idx, np.int64)
    n = int(np.prod(P.dims))
    sens = np.zeros(n * P.var_dim, np.float64)
    max_seeds = max(16, len(P.seed_index) + 16)
    so_i = np.zeros(max_seeds, np.int64)
    so_w = np.zeros(max_seeds, np.float64)
    values = np.ascontiguousarray(res["values"].ravel())
    ns = lib().fmo_backward_variation(ctypes.byref(P.struct), _ptr(values), _ptr(res["activeNeighs"]),
                                      len(idx), _ptr(idx), _ptr(wts), _ptr(sens), max_seeds,
                                      _ptr(so_i), _ptr(so_w))
    if ns < 0:
        raise RuntimeError("oracle backward variation failed")
    ns = min(int(ns), max_seeds)
    shape = P.dims + ((P.var_dim,) if P.var_dim > 1 else ())
    return sens.reshape(shape), so_i[:ns].copy(), so_w[:ns].copy()


def visibility(params: Dict, max_width: int):
    P = Problem(params)
    n = int(np.prod(P.dims))
    nb = P.nfwd + 2 * P.nsym
    vis = np.zeros((n, nb), np.uint8)
    if lib().fmo_visibility(ctypes.byref(P.struct), max_width, _ptr(vis)):
        raise RuntimeError("oracle visibility failed")
    return vis


def tti_norm(metric, h):
    """{tmin, tmax, optimDirection, Multiplier(tmin), Multiplier(tmax)} of one TTI metric element
    (14 values) at grid scales h (``TTINorm.hxx:62-87, 165-226``)."""
    m = np.ascontiguousarray(metric, np.float64)
    hh = np.ascontiguousarray(np.broadcast_to(np.asarray(h, float), (3,)))
    out = np.zeros(5)
    if lib().fmo_tti_norm(_ptr(m), _ptr(hh), _ptr(out)) != 0:
        raise ValueError("invalid TTI metric")
    return out


def tti_solve(params: Dict) -> Dict:
    """Semi-Lagrangian fast marching of a TTI3 ``params`` dictionary (RowMajor arrays)."""
    dims = tuple(int(round(d)) for d in np.asarray(params["dims"]).ravel())
    hs = np.asarray(params.get("gridScales", [params.get("gridScale", 1.0)] * 3), float)
    hs = np.ascontiguousarray(np.broadcast_to(hs, (3,)))
    origin = np.asarray(params.get("origin", np.zeros(3)), float)
    metric = np.ascontiguousarray(np.broadcast_to(np.asarray(params["metric"], float), dims + (14,)))
    sidx, sval = _seed_indices(params, lambda p: (np.asarray(p) - origin) / hs, dims, [0, 0, 0])
    n = int(np.prod(dims))
    values = np.empty(n)
    tact = np.empty(n)
    d = np.array(dims, np.int64)
    # stopping criteria (CommonStoppingCriteria.h:95-147) in a problem structure of their own
    stop, keep = _Problem(), []
    has_stop = False
    if "stopAtDistance" in params:
        stop.has_stop_at_distance, stop.stop_at_distance, has_stop = 1, float(params["stopAtDistance"]), True
    if "nMaxAccepted" in params:
        stop.n_max_accepted, has_stop = int(params["nMaxAccepted"]), True
    for key, fld in (("stopWhenAnyAccepted", "stop_any"), ("stopWhenAllAccepted", "stop_all")):
        if key in params:
            cells = []
            for q in np.atleast_2d(np.asarray(params[key], float)):
                i = np.floor((q - origin) / hs).astype(np.int64)
                if np.all((i >= 0) & (i < d)):
                    cells.append(int(np.ravel_multi_index(tuple(i), dims)))
            arr = np.ascontiguousarray(cells, np.int64)
            keep.append(arr)
            setattr(stop, "n" + fld, len(arr))
            setattr(stop, fld, _ptr(arr))
            has_stop = True
    # static factoring given as arrays (the reference's exported factoringValues / factoringGradients /
    # factoringIndexShift: adimensional gradients, a subdomain box when the shift is given)
    if "_factor" in params:
        fv, fg, shift = params["_factor"]
        fv = np.ascontiguousarray(fv, float)
        fg = np.ascontiguousarray(np.asarray(fg, float).reshape(fv.shape + (3,)))
        fm = np.ascontiguousarray((np.asarray(params["_factor_mask"]) != 0).astype(np.uint8) if "_factor_mask" in params
                                  else np.ones(fv.shape, np.uint8))
        keep += [fv, fg, fm]
        stop.fac_values, stop.fac_grads, stop.fac_mask = _ptr(fv), _ptr(fg), _ptr(fm)
        for a in range(3):
            stop.fac_lo[a] = int(shift[a]) if shift is not None else 0
            stop.fac_dims[a] = fv.shape[a]
        stop.fac_subdomain = 1 if shift is not None else 0
        has_stop = True
    nacc = lib().fmo_tti_fast_marching_stop(_ptr(d), _ptr(hs), _ptr(metric), len(sidx), _ptr(sidx), _ptr(sval),
                                            _ptr(values), _ptr(tact), ctypes.byref(stop) if has_stop else None)
    if nacc < 0:
        raise RuntimeError("oracle TTI fast marching failed")
    return {"values": values.reshape(dims), "activeNeighs": tact.reshape(dims), "nAccepted": int(nacc),
            "_tti": (d, hs, metric, origin), "_seeds": sidx, "_stop": (stop, keep) if has_stop else None}


def tti_prefix_solve(res: Dict) -> np.ndarray:
    """The TTI update of every cell recomputed from the finished values of a :func:`tti_solve`
    result, in the order-independent form that the parallel solver iterates to (each neighbour's
    acceptance triggering a solve over the neighbours at or below it, while below the result so
    far), with the same static factor. Equal to the values when fast marching's result is a fixed
    point of that form."""
    d, hs, metric, origin = res["_tti"]
    values = np.ascontiguousarray(res["values"].ravel(), float)
    seed = np.zeros(values.size, np.uint8)
    seed[res["_seeds"]] = 1
    out = np.empty_like(values)
    st = res["_stop"]
    rc = lib().fmo_tti_prefix_solve(_ptr(d), _ptr(hs), _ptr(metric), _ptr(values), _ptr(seed),
                                    ctypes.byref(st[0]) if st else None, _ptr(out))
    if rc != 0:
        raise RuntimeError("oracle TTI prefix solve failed")
    return out.reshape(res["values"].shape)


def tti_prefix_fixed_point(res: Dict, max_sweeps: int = 100000) -> np.ndarray:
    """The fixed point of the order-independent TTI update (:func:`tti_prefix_solve`) reached by
    Jacobi sweeps from the seeds of a :func:`tti_solve` result: what a parallel solver converges to.
    With static factoring it can differ from fast marching, whose corrected updates are taken in
    acceptance order; without it the two agree."""
    d, hs, metric, origin = res["_tti"]
    v = np.full(res["values"].size, np.inf)
    seed = np.zeros(v.size, np.uint8)
    seed[res["_seeds"]] = 1
    v[res["_seeds"]] = res["values"].ravel()[res["_seeds"]]
    st = res["_stop"]
    it = lib().fmo_tti_prefix_fixed_point(_ptr(d), _ptr(hs), _ptr(metric), _ptr(v), _ptr(seed),
                                          ctypes.byref(st[0]) if st else None, int(max_sweeps))
    if it < 0:
        raise RuntimeError("oracle TTI fixed point: no convergence")
    return v.reshape(res["values"].shape)


def tti_backward_variation(res: Dict, points, weights=None):
    """Reverse first variation of a :func:`tti_solve` result from weighted physical points.
    Returns (costSensitivity, seed indices, seed weights)."""
    d, hs, metric, origin = res["_tti"]
    dims = tuple(int(x) for x in d)
    pts = np.atleast_2d(np.asarray(points, float))
    w = np.ones(len(pts)) if weights is None else np.asarray(weights, float).ravel()
    idx = []
    for q in pts:
        i = np.floor((q - origin) / hs).astype(np.int64)
        idx.append(int(np.ravel_multi_index(tuple(i), dims)) if np.all((i >= 0) & (i < dims)) else -1)
    idx = np.asarray(idx, np.int64)
    values = np.ascontiguousarray(res["values"].ravel())
    tact = np.ascontiguousarray(res["activeNeighs"].ravel())
    sens = np.empty(values.size)
    cap = 1 << 16
    si = np.empty(cap, np.int64)
    sw = np.empty(cap)
    ns = lib().fmo_tti_backward_variation(_ptr(d), _ptr(hs), _ptr(metric), _ptr(values), _ptr(tact), len(idx),
                                          _ptr(idx), _ptr(np.ascontiguousarray(w)), _ptr(sens), cap, _ptr(si),
                                          _ptr(sw))
    if ns < 0:
        raise RuntimeError("oracle TTI backward variation failed")
    return sens.reshape(dims), si[:ns], sw[:ns]


def _geo_params(params: Dict, ndim: int):
    """geodesicStep, geodesicWeightThreshold, geodesicVolumeBound with the reference's defaults
    (``GeodesicDiscreteSolver.h:17-19``)."""
    return (float(_get(params, "geodesicStep", 0.25)), float(_get(params, "geodesicWeightThreshold", 0.001)),
            float(_get(params, "geodesicVolumeBound", 5.0 * 1.3 ** ndim)))


def _unoriented_tips(values, adim, dims, tips_u):
    """tips_Unoriented -> oriented dimensionless tips: among the angles at the cell centres, the one
    of smallest value, the last one on ties (``HFMInterface.hxx:499-521`` with ``:56-90``)."""
    out = []
    for q in np.atleast_2d(np.asarray(tips_u, float)):
        base = adim(np.array([q[0], q[1], 0.0]))
        best, vmin = None, math.inf
        for t in range(dims[2]):
            p = np.array([base[0], base[1], t + 0.5])
            i, j = int(math.floor(p[0])), int(math.floor(p[1]))
            if best is None:
                best = p
            if not (0 <= i < dims[0] and 0 <= j < dims[1]):
                continue
            v = values[i, j, t]
            if vmin < v:
                continue
            best, vmin = p, v
        out.append(best)
    return np.array(out)


def _run_discrete(fn, args, tips, step, thr, vb, ndim):
    tips = np.ascontiguousarray(np.atleast_2d(tips), np.float64)
    cap = 1 << 16
    while True:
        pts = np.empty((cap, ndim))
        lens = np.zeros(len(tips), np.int64)
        failed = np.zeros(len(tips), np.int32)
        extra = (step, thr) if vb is None else (step, thr, vb)
        n = fn(*args, len(tips), _ptr(tips), *extra, cap, _ptr(pts), _ptr(lens), _ptr(failed))
        if n == -2:
            cap *= 4
            continue
        if n < 0:
            raise RuntimeError("oracle geodesic extraction failed")
        return pts[:n].copy(), lens, failed


def geodesics(res: Dict, params: Dict) -> Dict:
    """Discrete geodesics of a :func:`solve` or :func:`tti_solve` result for the ``tips`` and
    ``tips_Unoriented`` keys of ``params``: geodesicPoints[_Unoriented] (physical coordinates,
    concatenated), geodesicLengths[_Unoriented] and the failure flags."""
    out = {}
    if "_tti" in res:
        d, hs, metric, origin = res["_tti"]
        ndim, scale, adim = 3, hs, (lambda p: (np.asarray(p, float) - origin) / hs)
        values = np.ascontiguousarray(res["values"].ravel())
        tact = np.ascontiguousarray(res["activeNeighs"].ravel())
        fn, args = lib().fmo_tti_geodesic_discrete, (_ptr(d), _ptr(hs), _ptr(metric), _ptr(values), _ptr(tact))
        dims = tuple(int(x) for x in d)
    else:
        P: Problem = res["problem"]
        ndim, scale, origin, adim, dims = P.ndim, P.scale, P.origin, P._adim, P.dims
        values = np.ascontiguousarray(res["values"].ravel())
        fn, args = lib().fmo_geodesic_discrete, (ctypes.byref(P.struct), _ptr(values), _ptr(res["activeNeighs"]))
    step, thr, vb = _geo_params(params, ndim)
    if params.get("geodesicSolver", "Discrete") == "ODE":
        # GeodesicODESolver.hxx:17-23: geodesicStep, geodesicCausalityTolerance (the target
        # tolerance of 6 is fixed when the solver is built, before the keys are read)
        caus = float(_get(params, "geodesicCausalityTolerance", 4.0))
        if "_tti" in res:
            sidx, _ = _seed_indices(params, adim, dims, [0, 0, 0])
            sidx = np.ascontiguousarray(sidx, np.int64)
            fn, args = lib().fmo_tti_geodesic_ode, args + (len(sidx), _ptr(sidx))
        else:
            fn = lib().fmo_geodesic_ode
        thr, vb = caus, None
    groups = []
    if "tips" in params:
        groups.append(("", np.array([adim(p) for p in np.atleast_2d(np.asarray(params["tips"], float))])))
    if "tips_Unoriented" in params and ndim == 3 and "_tti" not in res:
        groups.append(("_Unoriented", _unoriented_tips(res["values"], adim, dims, params["tips_Unoriented"])))
    for suffix, tips in groups:
        pts, lens, failed = _run_discrete(fn, args, tips, step, thr, vb, ndim)
        out["geodesicPoints" + suffix] = pts * scale + origin
        out["geodesicLengths" + suffix] = lens.astype(float)
        out["geodesicFailed" + suffix] = failed
    return out


def geodesic_flow(res: Dict) -> np.ndarray:
    """exportGeodesicFlow of a solve result: -ReDim of the Recompute flow at every cell, dims + (ndim,)."""
    if "_tti" in res:
        d, hs, metric, origin = res["_tti"]
        dims, scale = tuple(int(x) for x in d), hs
        values = np.ascontiguousarray(res["values"].ravel())
        tact = np.ascontiguousarray(res["activeNeighs"].ravel())
        flow = np.empty((values.size, 3))
        lib().fmo_tti_geodesic_flow(_ptr(d), _ptr(hs), _ptr(metric), _ptr(values), _ptr(tact), _ptr(flow), None, None)
    else:
        P: Problem = res["problem"]
        dims, scale = P.dims, P.scale
        values = np.ascontiguousarray(res["values"].ravel())
        flow = np.empty((values.size, P.ndim))
        lib().fmo_geodesic_flow(ctypes.byref(P.struct), _ptr(values), _ptr(res["activeNeighs"]), _ptr(flow), None, None)
    return (-(flow * scale)).reshape(dims + (len(dims),))


def forward_variation(res: Dict, params: Dict) -> np.ndarray:
    """valueVariation of a :func:`solve` or :func:`tti_solve` result for the ``costVariation`` and
    ``seedValueVariation`` keys of ``params`` (RowMajor): dims + (nVar,)
    (``FirstVariation.h:103-124, 389-429``)."""
    tti = "_tti" in res
    if tti:
        d, hs, metric, origin = res["_tti"]
        dims = tuple(int(x) for x in d)
        adim = lambda q: (np.asarray(q, float) - origin) / hs
        periodic = [0, 0, 0]
    else:
        P: Problem = res["problem"]
        dims, adim, periodic = P.dims, P._adim, P.periodic
    n = int(np.prod(dims))
    cost = None
    nvar = 0
    vd = 1 if tti else P.var_dim
    if "costVariation" in params:
        cost = np.ascontiguousarray(np.asarray(params["costVariation"], float).reshape(n, -1))
        nvar = cost.shape[1] // vd
    seedvar = None
    if "seedValueVariation" in params:
        seedvar = np.atleast_2d(np.asarray(params["seedValueVariation"], float))
        nvar = max(nvar, seedvar.shape[0])
    result = np.zeros((n, nvar))
    if seedvar is not None:
        seeds = np.atleast_2d(np.asarray(params["seeds"], float))
        if seeds.shape[0] != seedvar.shape[1]:
            raise ValueError("Error : Inconsistent size of seedValueVariation")
        for i, q in enumerate(seeds):
            idx = [int(math.floor(c)) for c in adim(q)]
            for a, m in enumerate(dims):
                if periodic[a]:
                    idx[a] %= m
            if all(0 <= idx[a] < dims[a] for a in range(len(dims))):
                result[np.ravel_multi_index(tuple(idx), dims)] = seedvar[:, i]
    values = np.ascontiguousarray(res["values"].ravel())
    if tti:
        tact = np.ascontiguousarray(res["activeNeighs"].ravel())
        rc = lib().fmo_tti_forward_variation(_ptr(d), _ptr(hs), _ptr(metric), _ptr(values), _ptr(tact), nvar,
                                             _ptr(cost), _ptr(result))
    else:
        rc = lib().fmo_forward_variation(ctypes.byref(P.struct), _ptr(values), _ptr(res["activeNeighs"]), nvar,
                                         _ptr(cost), _ptr(result))
    if rc != 0:
        raise RuntimeError("oracle forward variation failed")
    return result.reshape(dims + (nvar,))


# ------------------------------------------------------------------------------- ReedsShepp3

def rs3_stencil(ntheta: int, nphi: int, h: float, xi: float, eps: float, dual: bool = False,
                forward: bool = False):
    """Shared ReedsShepp3 stencils per class (theta, phi) = it * nphi + ip: offsets [ncls, 8, 5]
    (x, y, z, theta, phi) and weights [ncls, 8] (``Curvature3.h:37-58``); ``forward``: the
    ReedsSheppForward3 stencils, 6 forward differences then the 2 angular ones (``:79-95``)."""
    ncls = ntheta * nphi
    off = np.zeros((ncls, 8, 5), np.int8)
    w = np.zeros((ncls, 8))
    if forward:
        rc = lib().fmo_rsf3_stencil(ntheta, nphi, h, xi, eps, _ptr(off), _ptr(w))
    else:
        rc = lib().fmo_rs3_stencil(ntheta, nphi, h, xi, eps, int(bool(dual)), _ptr(off), _ptr(w))
    if rc != 0:
        raise RuntimeError("ObtuseSuperbase error in the ReedsShepp3 stencil")
    return off, w


def _rs3_seed_index(q, dims):
    """Index of an adimensionalized point: floor per axis, then the index periodization
    (``StaticFactoring.hxx:384-390``, ``PeriodicGrid.hxx:120-160``); None outside."""
    idx = [int(math.floor(c)) for c in q]
    if not all(0 <= idx[a] < dims[a] for a in range(3)):
        return None
    nt, nph = dims[3], dims[4]
    t = idx[3] % (2 * nt)
    if t >= nt:
        t = 2 * nt - t - 1
        idx[4] += nph // 2
    idx[3] = t
    idx[4] %= nph
    return int(np.ravel_multi_index(tuple(idx), dims))


def rs3_solve(params: Dict) -> Dict:
    """ReedsShepp3 / ReedsSheppForward3 fast marching on the CPU (``Curvature3.h:29-107``): values
    (dims), activeNeighs (uint64), nAccepted, MaxStencilWidth. Keys: model, dims (5), gridScale,
    origin (3), xi, eps, dual and projective (ReedsShepp3; projective: nphi = 4 ntheta instead of
    2 ntheta), speed or cost (scalar; (x, y, z); (theta, phi); or the full grid), seeds (n, 5),
    seedValues."""
    dims = tuple(int(round(d)) for d in np.asarray(params["dims"]).ravel())
    if len(dims) != 5:
        raise ValueError("ReedsShepp3 takes five dims")
    forward = params.get("model") == "ReedsSheppForward3"
    nt, nph = dims[3], dims[4]
    projective = bool(_get(params, "projective", 0.0)) and not forward
    if nph != (4 if projective else 2) * nt:
        raise ValueError("ReedsShepp3 setup error : inconsistent bundle dimensions")
    h = float(params["gridScale"])
    xi, eps = float(_get(params, "xi", 1.0)), float(_get(params, "eps", 0.1))
    dual = bool(_get(params, "dual", 0.0)) and not forward
    off, w = rs3_stencil(nt, nph, h, xi, eps, dual, forward)
    nfwd, nsym = (6, 2) if forward else (0, 8)
    if "speed" in params:
        sp = np.asarray(params["speed"], float)
    else:
        sp = 1.0 / np.asarray(params["cost"], float)
    if sp.ndim == 2:       # a field over (theta, phi)
        sp = sp.reshape((1, 1, 1, nt, nph))
    elif sp.ndim == 3:     # a field over (x, y, z)
        sp = sp.reshape(dims[:3] + (1, 1))
    mult = np.ascontiguousarray(np.broadcast_to(sp, dims), dtype=np.float64)
    ds = 2.0 * math.pi / nph
    origin = np.asarray(_get(params, "origin", np.zeros(3)), float).ravel()
    seen = {}
    if "seeds" in params:
        pts = np.atleast_2d(np.asarray(params["seeds"], float))
        vals = np.asarray(_get(params, "seedValues", np.zeros(len(pts))), float).ravel()
        for p, v in zip(pts, vals):
            q = [(p[0] - origin[0]) / h, (p[1] - origin[1]) / h, (p[2] - origin[2]) / h, p[3] / ds,
                 (p[4] + ds / 2.0) / ds]
            lin = _rs3_seed_index(q, dims)
            if lin is not None:
                seen.setdefault(lin, float(v))
    keys = sorted(seen)
    sidx = np.array(keys, np.int64)
    sval = np.array([seen[k] for k in keys], float)
    n = int(np.prod(dims))
    values = np.empty(n)
    active = np.zeros(n, np.uint64)
    mw = ctypes.c_int(0)
    d = np.array(dims, np.int64)
    nacc = lib().fmo_s2_fast_marching(_ptr(d), nfwd, nsym, _ptr(off), _ptr(w), _ptr(mult), len(sidx), _ptr(sidx),
                                      _ptr(sval), _ptr(values), _ptr(active), ctypes.byref(mw))
    if nacc < 0:
        raise RuntimeError("oracle ReedsShepp3 fast marching failed")
    return {"values": values.reshape(dims), "activeNeighs": active, "nAccepted": int(nacc),
            "MaxStencilWidth": int(mw.value)}
