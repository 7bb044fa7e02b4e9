"""The ALE remap step without a GPU: the oracle's invariants and golden vectors,
and the C-ABI (include/ale_b200.h) — every declared symbol exported, invalid
arguments rejected before the device is touched.

The golden vectors (tests/golden/ale_*.npz) hold seeded inputs and the outputs of
the reference's own CUDA launcher `ale_remap_cuda` (ale_remap/ale_kernel.cu,
faithful form, built from the reference sources with FMA contraction off;
tests/golden/make_ale_golden.py). The oracle must reproduce every output array
after every step bit for bit.
"""

import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

from more_benchmarks_dc_ocean_b200 import ale_inputs as AI
from oracle import ale_oracle as AO

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ale_b200.h")
GOLDEN = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "ale_*.npz")))


def _declared():
    return re.findall(r"^ALE_B200_API\s+[\w\s\*]*?\b(\w+)\s*\(", open(HEADER).read(), flags=re.M)


def test_header_declares_the_reference_launchers():
    names = _declared()
    for n in ("ale_remap_cuda", "ale_remap_opt", "cuda_sync", "ale_b200_remap_step", "ale_b200_last_error"):
        assert n in names


def test_every_declared_symbol_is_exported(redi_lib):
    from more_benchmarks_dc_ocean_b200 import ale_remap as A

    L = A.lib()
    missing = [n for n in _declared() if not hasattr(L, n)]
    assert not missing, missing


def test_invalid_arguments_rejected_without_a_device(redi_lib):
    from more_benchmarks_dc_ocean_b200 import ale_remap as A

    L = A.lib()
    assert L.ale_b200_remap_step(None, None) == A.E_ARG
    a = A.StepArgs()
    a.nx, a.ny, a.nz, a.method = 4, 3, 129, 3
    assert L.ale_b200_remap_step(C.byref(a), None) == A.E_ARG
    assert "NZ_MAX" in A.last_error()
    a.nz = 5
    for m in (4, 5):
        a.method = m
        assert L.ale_b200_remap_step(C.byref(a), None) == A.E_UNSUPPORTED
    a.method = 3
    assert L.ale_b200_remap_step(C.byref(a), None) == A.E_ARG  # NULL arrays
    a.nx = 0
    assert L.ale_b200_remap_step(C.byref(a), None) == A.E_ARG


def test_compat_launchers_report_invalid_arguments(redi_lib, capfd):
    from more_benchmarks_dc_ocean_b200 import ale_remap as A

    A.ale_remap_cuda(4, 4, 300, 3, 0, *([None] * 15))
    A.ale_remap_opt(0, 4, 5, *([None] * 13))
    err = capfd.readouterr().err
    assert "ale_remap_cuda" in err and "ale_remap_opt" in err


@pytest.mark.parametrize("method", [AI.REMAP_PCM, AI.REMAP_PLM, AI.REMAP_PPM])
def test_remap_conserves_column_content(method):
    """sum_k hTr is unchanged in every column where no source layer is floored away
    (h_old > H_FLOOR everywhere), and the budgets record exactly the change."""
    p = AI.random_case(18, 14, 11, 11, vanished=0.0, zero_targets=1, method=method, budgets_nonzero=False)
    p.h_layer[p.h_layer < 1e-3] = 1e-3
    T0 = [t.sum(0).copy() for t in p.tracers]
    q = p.copy()
    AO.step(q, 1)
    for n, (a, b) in enumerate(zip(T0, q.tracers)):
        rel = np.abs(b.sum(0) - a).max() / np.abs(a).max()
        assert rel < 1e-12, (method, n, rel)
    assert np.abs(q.heat_budget.sum(0)).max() <= 1e-9 * np.abs(p.tracers[0]).sum(0).max()
    np.testing.assert_array_equal(q.h_layer, q.target_h)
    np.testing.assert_array_equal(q.h_old, p.h_layer)


def test_target_and_eta_follow_the_zstar_formula():
    p = AI.reference_ic(30, 20, 10)
    q = p.copy()
    AO.step(q, 1)
    s = np.zeros((p.ny, p.nx))
    for k in range(p.nz):
        s = s + p.h_layer[k]
    np.testing.assert_array_equal(q.total_h, s)
    np.testing.assert_array_equal(q.h_ref, s - p.bt_eta)
    for k in range(p.nz):
        np.testing.assert_array_equal(q.target_h[k], (q.h_ref + p.bt_eta) * p.dsig[k])
    e = -p.bt_H_ref
    for k in range(p.nz):
        e = e + q.h_layer[k]
    np.testing.assert_array_equal(q.bt_eta, e)


def test_second_step_is_a_fixed_point_for_thicknesses():
    """The zstar target depends only on the column total, so a second step leaves h unchanged."""
    p = AI.reference_ic(24, 18, 9)
    AO.step(p, 1)
    h1 = p.h_layer.copy()
    AO.step(p, 1)
    assert np.allclose(p.h_layer, h1, rtol=1e-13, atol=1e-12)


def test_golden_fixtures_present():
    assert len(GOLDEN) >= 6, "ALE golden fixtures missing: run tests/golden/make_ale_golden.py on a GPU"


def _problem(z) -> AI.AleProblem:
    g = lambda k: z["in_" + k].copy()  # noqa: E731
    return AI.AleProblem(str(z["name"]), int(z["nx"]), int(z["ny"]), int(z["nz"]), g("h_layer"),
                         [g("tracer0"), g("tracer1")], g("u"), g("v"), g("mass_budget"), g("heat_budget"),
                         g("salt_budget"), g("bt_eta"), g("bt_H_ref"), g("dsig"))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(g)[:-4] for g in GOLDEN])
def test_oracle_matches_reference_cuda(path):
    z = np.load(path)
    p = _problem(z)
    for s in range(int(z["nsteps"])):
        AO.step(p, 1)
        got = p.arrays()
        for k in got:
            key = f"ref_step{s + 1}_{k}"
            if key in z.files:
                assert np.array_equal(got[k], z[key]), f"{k} after step {s + 1}"
