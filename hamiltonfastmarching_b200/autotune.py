"""Autotuner of the solver's schedule: tile shape, local sweeps per activation, queue policy.

The tiled solver's speed depends on three choices that do not change its result (the fixed point
of the local solves): the shape of the 64-cell tiles (`tileShape`), the number of local sweeps a
tile runs per activation (`tileSweeps`), and the queue policy (`tileOrdering` with the band limits
`bandLo`/`bandHi`, or plain FIFO rounds). The best choice depends on the model, the precision, the
grid size and the GPU. :class:`Autotuner` measures candidates on a sample of instances (GPU time of
a batched solve, best of `repeats`), searches coordinate by coordinate, and keeps the winners in a
JSON table keyed by (model, precision, size class, device). :meth:`Autotuner.apply` fills the
tuned keys of an ``hfmIn`` dictionary that does not set them.
"""
from __future__ import annotations

import json
import math
import os
from typing import Dict, List, Optional

import numpy as np

from . import run_batch

__all__ = ["Autotuner", "family_key", "SPACE"]

# Candidates per parameter; tile shapes per domain kind (extents per axis, 64 cells).
SPACE = {
    "tileSweeps": [1, 2, 3, 4, 6],
    "queue": [("band", 0.5, 4.0), ("band", 1.0, 4.0), ("band", 2.0, 8.0), ("band", 4.0, 16.0), ("fifo", None, None)],
    "tileShape": {
        "2d": [(8, 8), (16, 4), (4, 16)],
        "3d": [(4, 4, 4), (8, 4, 2), (2, 4, 8), (4, 8, 2)],
        "lifted": [(4, 4, 4), (8, 8, 1), (2, 2, 16), (8, 4, 2)],
        # ReedsShepp3: (x, y, (z, theta, phi)) as the solver holds the sphere bundle
        "sphere": [(8, 8, 1), (4, 4, 4), (16, 4, 1), (8, 4, 2)],
    },
}
# The library's default schedule per model (default_schedule in the solver), the search's start.
DEFAULT = {
    "Riemann3": {"tileSweeps": 2, "queue": ("band", 0.5, 4.0)},
    "Riemann2": {"tileSweeps": 3, "queue": ("band", 2.0, 8.0)},
    "Isotropic2": {"tileSweeps": 3, "queue": ("band", 2.0, 8.0)},
    "Isotropic3": {"tileSweeps": 2, "queue": ("band", 0.5, 4.0)},
    "Diagonal2": {"tileSweeps": 3, "queue": ("band", 2.0, 8.0)},
    "Diagonal3": {"tileSweeps": 2, "queue": ("band", 0.5, 4.0)},
    "ReedsShepp2": {"tileSweeps": 4, "queue": ("band", 2.0, 8.0)},
    "ReedsSheppForward2": {"tileSweeps": 4, "queue": ("band", 2.0, 8.0)},
    "Elastica2": {"tileSweeps": 2, "queue": ("band", 4.0, 16.0)},
    "TTI3": {"tileSweeps": 1, "queue": ("band", 1.0, 4.0)},
    "ReedsShepp3": {"tileSweeps": 1, "queue": ("band", 4.0, 16.0)},
    "ReedsSheppForward3": {"tileSweeps": 1, "queue": ("band", 4.0, 16.0)},
}
_LIFTED = ("ReedsShepp2", "ReedsSheppForward2", "Elastica2")


def _domain_kind(params: Dict) -> str:
    if params["model"] in _LIFTED:
        return "lifted"
    if params["model"] in ("ReedsShepp3", "ReedsSheppForward3"):
        return "sphere"
    return "2d" if len(np.asarray(params["dims"]).ravel()) == 2 else "3d"


def family_key(params: Dict, device: str = "") -> str:
    """(model, precision, size class, device): size class = log2 of the cell count, rounded."""
    cells = float(np.prod(np.asarray(params["dims"], float)))
    size = int(round(math.log2(max(cells, 1.0))))
    prec = params.get("solverPrecision", "float64")
    return f"{params['model']}|{prec}|2^{size}|{device}"


def _device_name() -> str:
    try:
        import torch
        if torch.cuda.is_available():
            return torch.cuda.get_device_name(0)
    except Exception:
        pass
    return "cuda"


def _with(params: Dict, cfg: Dict) -> Dict:
    p = dict(params)
    p["verbosity"] = 0.0
    p["tileSweeps"] = float(cfg["tileSweeps"])
    kind, lo, hi = cfg["queue"]
    p["tileOrdering"] = 1.0 if kind == "band" else 0.0
    if kind == "band":
        p["bandLo"], p["bandHi"] = float(lo), float(hi)
    if cfg.get("tileShape") is not None:
        p["tileShape"] = np.asarray(cfg["tileShape"], float)
    return p


class Autotuner:
    def __init__(self, path: Optional[str] = None, repeats: int = 2, device: Optional[str] = None):
        self.path = path
        self.repeats = repeats
        self.device = device if device is not None else _device_name()
        self.table: Dict[str, Dict] = {}
        if path and os.path.exists(path):
            with open(path) as f:
                self.table = json.load(f)
        self.trials: List[Dict] = []

    def measure(self, cases: List[Dict], cfg: Dict) -> float:
        """GPU time (solve + stencils) of one batched solve of `cases` under `cfg`, best of repeats;
        +inf if the configuration fails (e.g. a dependency table overflows)."""
        best = math.inf
        for _ in range(self.repeats):
            try:
                outs = run_batch([_with(p, cfg) for p in cases])
            except Exception:
                return math.inf
            t = outs[0]["GPUSolveTime"] + outs[0]["GPUStencilTime"]
            best = min(best, t)
        self.trials.append({"cfg": {k: (list(v) if isinstance(v, tuple) else v) for k, v in cfg.items()},
                            "seconds": best})
        return best

    def tune(self, cases: List[Dict], sweeps: int = 2, params=("tileShape", "tileSweeps", "queue")) -> Dict:
        """Coordinate search over `params` (of tile shape, sweeps and queue policy) on a sample of
        instances of one family; returns (and records) the best configuration and its time against
        the defaults. A candidate replaces the incumbent only if it is 2% faster."""
        kind = _domain_kind(cases[0])
        cfg = dict(DEFAULT[cases[0]["model"]], tileShape=SPACE["tileShape"][kind][0])
        base = self.measure(cases, cfg)
        best_t = base
        for _ in range(sweeps):
            improved = False
            for name, values in (("tileShape", SPACE["tileShape"][kind]), ("tileSweeps", SPACE["tileSweeps"]),
                                 ("queue", SPACE["queue"])):
                if name not in params:
                    continue
                for v in values:
                    if v == cfg[name]:
                        continue
                    trial = dict(cfg, **{name: v})
                    t = self.measure(cases, trial)
                    if t < best_t * 0.98:
                        best_t, cfg, improved = t, trial, True
            if not improved:
                break
        key = family_key(cases[0], self.device)
        result = {"tileShape": list(cfg["tileShape"]), "tileSweeps": cfg["tileSweeps"],
                  "queue": list(cfg["queue"]), "seconds": best_t, "default_seconds": base}
        self.table[key] = result
        if self.path:
            with open(self.path, "w") as f:
                json.dump(self.table, f, indent=1, sort_keys=True)
        return result

    def lookup(self, params: Dict) -> Optional[Dict]:
        """Entry of the family of `params`; else the nearest size class of the same model,
        precision and device."""
        key = family_key(params, self.device)
        if key in self.table:
            return self.table[key]
        model, prec, size, dev = key.split("|")
        s0 = int(size[2:])
        best, dist = None, None
        for k, v in self.table.items():
            m, pr, sz, d = k.split("|")
            if (m, pr, d) != (model, prec, dev):
                continue
            dd = abs(int(sz[2:]) - s0)
            if dist is None or dd < dist:
                best, dist = v, dd
        return best

    def apply(self, params: Dict) -> Dict:
        """`params` with the tuned keys of its family filled in where it does not set them."""
        t = self.lookup(params)
        if t is None:
            return params
        p = dict(params)
        kind, lo, hi = t["queue"]
        tuned = {"tileSweeps": float(t["tileSweeps"]), "tileShape": np.asarray(t["tileShape"], float),
                 "tileOrdering": 1.0 if kind == "band" else 0.0}
        if kind == "band":
            tuned["bandLo"], tuned["bandHi"] = float(lo), float(hi)
        for k, v in tuned.items():
            p.setdefault(k, v)
        return p
