"""Autotuner table logic (CPU): keys, nearest-size lookup, filling of untuned keys only."""
import numpy as np

from hamiltonfastmarching_b200.autotune import Autotuner, family_key
from hamiltonfastmarching_b200 import workloads as W


def test_family_key_and_apply(tmp_path):
    at = Autotuner(path=None, device="B200")
    p = W.riemann2_case(64)
    p["solverPrecision"] = "float32"
    assert family_key(p, "B200") == "Riemann2|float32|2^12|B200"
    at.table["Riemann2|float32|2^12|B200"] = {"tileShape": [16, 4], "tileSweeps": 3, "queue": ["band", 1.0, 4.0]}
    at.table["Riemann2|float32|2^20|B200"] = {"tileShape": [8, 8], "tileSweeps": 6, "queue": ["fifo", None, None]}
    q = at.apply(p)
    assert list(q["tileShape"]) == [16, 4] and q["tileSweeps"] == 3 and q["bandLo"] == 1.0 and q["tileOrdering"] == 1.0
    big = W.riemann2_case(900)
    big["solverPrecision"] = "float32"
    q = at.apply(big)  # nearest size class: 2^20
    assert q["tileSweeps"] == 6 and q["tileOrdering"] == 0.0 and "bandLo" not in q
    p["tileSweeps"] = 8.0  # explicit keys win
    assert at.apply(p)["tileSweeps"] == 8.0
    other = W.riemann2_case(64)  # float64: no entry
    assert at.apply(other) is other
