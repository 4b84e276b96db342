"""Parity of the CUDA solve path (through the C ABI) with the reference and the C oracle.

Tolerances: FP64 arrival times within 1e-10 relative max-norm of the reference (the solver
reproduces fast marching's accumulation order, so most cells are bit-identical); stencil-derived
integers (nAccepted, MaxStencilWidth) exact; activeNeighs equal except where a symmetric
difference's two neighbours hold exactly the same value (fast marching then takes the side it
accepted first, this solver the +e side); FP32 path within 1e-5 relative of FP64.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN_SOLVES, GOLDEN_STENCILS, ROOT, load_golden
import hamiltonfastmarching_b200 as H
from hamiltonfastmarching_b200 import workloads as W
from oracle import oracle as O
from oracle.refrun import read_output, write_input

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-10


def rel_err(a, b):
    a, b = np.asarray(a), np.asarray(b)
    assert np.array_equal(np.isinf(a), np.isinf(b)), "reached sets differ"
    fin = np.isfinite(a)
    if not fin.any():
        return 0.0
    return float(np.max(np.abs(a[fin] - b[fin])) / max(np.max(np.abs(a[fin])), 1e-300))


def gpu_solve(params, **extra):
    p = dict(params)
    p.setdefault("verbosity", 0.0)
    p.update(extra)
    return H.run(p)


@pytest.mark.parametrize("name", GOLDEN_SOLVES + GOLDEN_STENCILS)
def test_golden_values(name):
    params, ref, _ = load_golden(name)
    out = gpu_solve(params)
    assert rel_err(ref["values"], out["values"]) <= FP64_RTOL
    assert int(out["nAccepted"]) == int(ref["nAccepted"])
    assert int(out["MaxStencilWidth"]) == int(ref["MaxStencilWidth"])
    same = np.mean(ref["values"] == out["values"])
    assert same > 0.99, f"only {same:.4f} of the cells are bit-identical"
    act_ref = ref["activeNeighs"].astype(np.uint64)
    act = out["activeNeighs"].astype(np.uint64)
    untied = untied_active_differences(params, ref["values"], act_ref, act)
    assert not untied, f"activeNeighs differ away from exact ties at cells {untied[:10]}"


def stencil_offsets_per_cell(params):
    """(nfwd, offsets [N][nfwd+nsym][ndim]) of the stencil each cell of `params` uses."""
    model = params["model"]
    dims = [int(d) for d in params["dims"]]
    if model.startswith("Riemann"):
        out = gpu_solve(params, exportStencils=1.0, exportValues=0.0)
        nk = 3 if len(dims) == 2 else 6
        return 0, out["stencilOffsets"].reshape(-1, nk, len(dims)).astype(np.int64)
    off, _ = O.curvature2_table(model, dims[2], float(params["gridScale"]), float(params.get("xi", 1.0)),
                                float(params.get("eps", 0.1)), bool(params.get("projective", 0.0)))
    nfwd = {"ReedsShepp2": 0, "ReedsSheppForward2": 3, "Elastica2": 27, "Dubins2": 12}[model]
    theta = np.arange(int(np.prod(dims))) % dims[2]
    return nfwd, off[theta].astype(np.int64)


def untied_active_differences(params, values, act_ref, act):
    """Cells whose activeNeighs differ other than by the side of an exactly tied symmetric pair."""
    bad = np.flatnonzero(act_ref.ravel() != act.ravel())
    if len(bad) == 0:
        return []
    nfwd, offs = stencil_offsets_per_cell(params)
    dims = values.shape
    periodic = [False] * (len(dims) - 1) + [params["model"] in ("ReedsShepp2", "ReedsSheppForward2", "Elastica2",
                                                                 "Dubins2")]
    v = values.ravel()

    def value_at(x, e):
        idx = list(np.unravel_index(x, dims))
        for a in range(len(dims)):
            idx[a] += int(e[a])
            if periodic[a]:
                idx[a] %= dims[a]
            elif not 0 <= idx[a] < dims[a]:
                return np.inf
        return v[np.ravel_multi_index(idx, dims)]

    untied = []
    for x in bad:
        r, o = int(act_ref.ravel()[x]), int(act.ravel()[x])
        fmask = (1 << nfwd) - 1
        nsym = offs.shape[1] - nfwd
        ok = (r & fmask) == (o & fmask) and (r >> (nfwd + 2 * nsym)) == (o >> (nfwd + 2 * nsym))
        for j in range(nsym):
            rb, ob = (r >> (nfwd + 2 * j)) & 3, (o >> (nfwd + 2 * j)) & 3
            if rb == ob:
                continue
            e = offs[x, nfwd + j]
            ok = ok and rb in (1, 2) and ob in (1, 2) and value_at(x, e) == value_at(x, -e)
        if not ok:
            untied.append(int(x))
    return untied


@pytest.mark.parametrize("name", GOLDEN_SOLVES)
def test_golden_sensitivity(name):
    params, ref, _ = load_golden(name)
    if "costSensitivity_0" not in ref:
        pytest.skip("fixture has no inspectSensitivity group")
    out = gpu_solve(params)
    a, b = ref["costSensitivity_0"], out["costSensitivity_0"]
    assert np.max(np.abs(a - b)) <= FP64_RTOL * np.max(np.abs(a))
    sr, so = ref["seedSensitivity_0"], out["seedSensitivity_0"]
    assert sr.shape == so.shape
    np.testing.assert_allclose(so, sr, rtol=1e-10, atol=0)


@pytest.mark.parametrize("case", ["riemann2_256", "riemann3_40_walls", "rs2_64x36", "elastica2_48x30", "rsf2_64x36"])
def test_oracle_parity_larger(case):
    if case == "riemann2_256":
        p = W.riemann2_case(256)
    elif case == "riemann3_40_walls":
        p = W.riemann3_case(40)
    elif case == "rs2_64x36":
        p = W.curvature2_case(64, 36, "ReedsShepp2")
    elif case == "rsf2_64x36":
        p = W.curvature2_case(64, 36, "ReedsSheppForward2")
    else:
        p = W.curvature2_case(48, 30, "Elastica2")
    ora = O.solve(p)
    out = gpu_solve(p)
    assert rel_err(ora["values"], out["values"]) <= FP64_RTOL
    assert int(out["nAccepted"]) == ora["nAccepted"]


@pytest.mark.parametrize("case", ["riemann2_128", "riemann3_32_walls", "rs2_48x30"])
def test_fp32_path_close_to_fp64(case):
    p = {"riemann2_128": lambda: W.riemann2_case(128),
         "riemann3_32_walls": lambda: W.riemann3_case(32, n_spheres=10, n_seeds=4),
         "rs2_48x30": lambda: W.curvature2_case(48, 30, "ReedsShepp2")}[case]()
    o64 = gpu_solve(p)
    o32 = gpu_solve(p, solverPrecision="float32")
    assert rel_err(o64["values"], o32["values"]) <= 1e-5


def test_yxz_ordering_default_of_python_binding():
    """HFMIO defaults to YXZ_RowMajor like the reference Python binding: arrays are transposed."""
    p = W.riemann2_case(48, aniso=8.0, seed=3)
    ref = gpu_solve(p)["values"]
    io = H.HFMIO()  # YXZ_RowMajor
    q = dict(p)
    del q["arrayOrdering"]
    q["metric"] = np.ascontiguousarray(np.transpose(p["metric"], (1, 0, 2)))
    q["verbosity"] = 0.0
    io.set_dict(q)
    io.run()
    assert rel_err(ref.T, io.get_array("values")) <= 1e-12


def test_non_spd_metric_is_an_error():
    p = W.riemann2_case(16)
    p["metric"] = p["metric"].copy()
    p["metric"][3, 4] = [1.0, 2.0, 1.0]   # determinant < 0
    with pytest.raises(H.PyExp) as e:
        gpu_solve(p)
    assert e.value.code == 2


def test_cli_matches_library(tmp_path):
    exe = os.path.join(ROOT, "hamiltonfastmarching_b200", "bin", "FileHFM_b200")
    params, ref, _ = load_golden("riemann3_16_walls")
    write_input(params, str(tmp_path / "input"))
    r = subprocess.run([exe, str(tmp_path / "input"), str(tmp_path / "output")], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    out = read_output(str(tmp_path / "output"))
    assert rel_err(ref["values"], out["values"]) <= FP64_RTOL
    assert out["nAccepted"] == ref["nAccepted"]
    link = tmp_path / "FileHFM_Riemann2"
    os.symlink(exe, link)
    r = subprocess.run([str(link), str(tmp_path / "input"), str(tmp_path / "o2")], capture_output=True, text=True)
    assert r.returncode != 0 and "Executable applies to Riemann2" in r.stdout


def test_repeatable_and_seeds_fixed():
    p = W.riemann3_case(32, n_spheres=8, n_seeds=5)
    a = gpu_solve(p)["values"]
    b = gpu_solve(p)["values"]
    assert rel_err(a, b) <= 1e-12  # the schedule may differ between runs: equal up to rounding
    P = O.Problem(p)
    np.testing.assert_array_equal(a.ravel()[P.seed_index], 0.0)


def test_device_entry_point_matches_host_api():
    """hfm_solve_riemann_device (inputs and output in device memory) equals HFMIO.run."""
    import ctypes
    import torch
    from hamiltonfastmarching_b200 import _lib
    p = W.riemann3_case(40, n_spheres=6, n_seeds=4)
    ref = gpu_solve(p)
    n = 40
    metric = torch.from_numpy(np.ascontiguousarray(p["metric"].reshape(-1, 6))).cuda()
    walls = torch.from_numpy(np.ascontiguousarray((p["walls"] != 0).astype(np.uint8).ravel())).cuda()
    values = torch.empty(n ** 3, dtype=torch.float64, device="cuda")
    ijk = np.floor(p["seeds"] / p["gridScale"]).astype(np.int64)
    sidx = np.ascontiguousarray(np.ravel_multi_index(ijk.T, (n, n, n)).astype(np.int64))
    sval = np.zeros(len(sidx))
    a = _lib.RiemannDeviceArgs()
    a.ndim = 3
    for i in range(3):
        a.dims[i] = n
        a.grid_scale[i] = p["gridScale"]
    a.precision = 64
    a.metric, a.walls, a.values = metric.data_ptr(), walls.data_ptr(), values.data_ptr()
    a.nseeds, a.seed_index, a.seed_value = len(sidx), sidx.ctypes.data, sval.ctypes.data
    a.stream = torch.cuda.current_stream().cuda_stream
    st = _lib.SolveStats()
    err = ctypes.create_string_buffer(256)
    assert _lib.load().hfm_solve_riemann_device(ctypes.byref(a), ctypes.byref(st), err, 256) == 0, err.value
    torch.cuda.synchronize()
    assert rel_err(ref["values"], values.cpu().numpy().reshape(n, n, n)) <= 1e-12
    assert st.n_accepted == int(ref["nAccepted"])
