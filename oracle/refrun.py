"""Run the reference's own FileHFM executables (built by ``make -C oracle ref`` into ``oracle/_ref``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, the golden-vector script, ``bench.py``'s CPU
baseline leg and ``__graft_entry__.smoke()`` as the checker. Never used by the product path.

The file pair format (``<prefix>_Format.txt`` + raw float64 ``<prefix>_Data.dat``) follows the
reference's reader/writer (``JMM_CPPLibs/Output/FileIO.hxx:7-132``): per key one line with the
name, one with the depth (-1 = string, 0 = scalar, d = array), d lines of dimensions, a blank line.
"""
from __future__ import annotations

import os
import subprocess
import tempfile
from typing import Dict

import numpy as np

REF_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref")


def ref_executable(model: str) -> str:
    return os.path.join(REF_DIR, "FileHFM_" + model)


def have_reference(model: str) -> bool:
    return os.access(ref_executable(model), os.X_OK)


def write_input(params: Dict, prefix: str) -> None:
    chunks = []
    with open(prefix + "_Format.txt", "w") as f:
        for key, val in params.items():
            if isinstance(val, str):
                f.write(f"{key}\n-1\n{val}\n\n")
            elif np.isscalar(val) or (isinstance(val, np.ndarray) and val.ndim == 0):
                f.write(f"{key}\n0\n\n")
                chunks.append(np.array([float(val)]))
            else:
                arr = np.asarray(val, dtype=np.float64)
                f.write(f"{key}\n{arr.ndim}\n")
                for d in arr.shape:
                    f.write(f"{d}\n")
                f.write("\n")
                chunks.append(arr.ravel())
    data = np.concatenate(chunks) if chunks else np.zeros(0)
    data.astype("<f8").tofile(prefix + "_Data.dat")


def read_output(prefix: str) -> Dict:
    data = np.fromfile(prefix + "_Data.dat", dtype="<f8")
    out, pos = {}, 0
    with open(prefix + "_Format.txt") as f:
        while True:
            key = f.readline().strip()
            if not key:
                break
            depth = int(f.readline())
            if depth == -1:
                out[key] = f.readline().strip()
            elif depth == 0:
                out[key] = float(data[pos])
                pos += 1
            else:
                dims = [int(f.readline()) for _ in range(depth)]
                size = int(np.prod(dims))
                out[key] = data[pos:pos + size].reshape(dims).copy()
                pos += size
            f.readline()
    return out


def run_reference(params: Dict, model: str = None, timeout: float = 3600.0) -> Dict:
    """Solve ``params`` with the reference FileHFM_<model> and return its output dictionary.

    Adds ``retcode`` and ``log``; raises ``RuntimeError`` if the executable is missing.
    """
    model = model or params["model"]
    exe = ref_executable(model)
    if not os.access(exe, os.X_OK):
        raise RuntimeError(f"reference executable {exe} not built (make -C oracle ref)")
    with tempfile.TemporaryDirectory(prefix="hfmref_") as tmp:
        ip, op = os.path.join(tmp, "input"), os.path.join(tmp, "output")
        write_input(params, ip)
        proc = subprocess.run([exe, ip, op], capture_output=True, text=True, timeout=timeout)
        out = read_output(op) if os.path.exists(op + "_Format.txt") else {}
        out["retcode"] = proc.returncode
        out["log"] = proc.stdout + proc.stderr
    return out
