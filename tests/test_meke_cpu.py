"""The MEKE step without a GPU: the oracle's invariants and golden vectors, and
the C-ABI (include/meke_b200.h) — every declared symbol exported, invalid
arguments rejected before the device is touched.

The golden vectors (tests/golden/meke_*.npz) hold seeded inputs and the outputs
of the reference's own CUDA launcher `meke_cuda_launch` mode 0 (the faithful
16-kernel form, meke/meke_kernel.cu, built from the reference sources with FMA
contraction off by oracle/ref_build.sh; tests/golden/make_meke_golden.py). The
oracle must reproduce every output array after every step bit for bit.
"""

import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

from more_benchmarks_dc_ocean_b200 import meke_inputs as MI
from oracle import meke_oracle as MO

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "meke_b200.h")
GOLDEN = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "meke_*.npz")))


def _declared():
    return re.findall(r"^MEKE_B200_API\s+[\w\s\*]*?\b(\w+)\s*\(", open(HEADER).read(), flags=re.M)


def test_header_declares_the_reference_launchers():
    names = _declared()
    for n in ("meke_cuda_launch", "meke_cuda_graph_reset", "meke_opt_launch", "meke_opt_launch_flat",
              "meke_b200_create", "meke_b200_step", "meke_b200_destroy"):
        assert n in names


def test_every_declared_symbol_is_exported(redi_lib):
    from more_benchmarks_dc_ocean_b200 import ocean_meke as M

    L = M.lib()
    missing = [n for n in _declared() if not hasattr(L, n)]
    assert not missing, missing


def test_args_struct_layout_matches_the_reference():
    """struct MekeArgs: 30 pointers, 3 ints, 23 doubles, 1 int (meke/meke_args.h:38-52)."""
    from more_benchmarks_dc_ocean_b200 import ocean_meke as M

    f = M.MekeArgs._fields_
    assert [n for n, _ in f[:30]] == list(M._PTRS)
    assert [n for n, _ in f[30:33]] == ["nx", "ny", "nz"]
    assert len(f) == 30 + 3 + 23 + 1 and f[-1][0] == "backscatter"
    assert C.sizeof(M.MekeArgs) == 30 * 8 + 3 * 4 + 4 + 23 * 8 + 8


def test_invalid_arguments_rejected_without_a_device(redi_lib):
    from more_benchmarks_dc_ocean_b200 import ocean_meke as M

    L = M.lib()
    h = C.c_void_p()
    assert L.meke_b200_create(0, 5, 3, C.byref(h)) == M.E_ARG
    assert L.meke_b200_create(5, 5, -1, C.byref(h)) == M.E_ARG
    assert L.meke_b200_create(5, 5, 3, None) == M.E_ARG
    assert L.meke_b200_create(70000, 70000, 3, C.byref(h)) == M.E_ARG
    assert "too large" in M.last_error()
    assert L.meke_b200_step(None, None, None, None) == M.E_ARG
    a = M.MekeArgs()
    a.nx, a.ny, a.nz = 4, 4, 2
    assert L.meke_b200_step(None, C.byref(a), None, None) == M.E_ARG
    assert "NULL" in M.last_error()
    assert L.meke_b200_destroy(None) == M.OK


def test_compat_launcher_reports_invalid_arguments(redi_lib, capfd):
    from more_benchmarks_dc_ocean_b200 import ocean_meke as M

    a = M.MekeArgs()
    a.nx, a.ny, a.nz = 0, 4, 2
    M.meke_cuda_launch(a, 0)
    M.meke_opt_launch(a, None)
    err = capfd.readouterr().err
    assert "meke_cuda_launch" in err and "meke_opt_launch" in err


def test_reference_ic_invariants():
    """The reference driver's configuration is degenerate (meke/drivers/cpp_main.cu:36-45):
    le == 0, kh_diff == 0, bottom_fac2 == barotr_fac2 == 1 exactly."""
    p = MI.reference_ic(60, 40, 7)
    MO.step(p, 2)
    a = p.arrays
    assert not a["le"].any() and not a["kh_diff"].any() and not a["ku"].any()
    assert (a["bottom_fac2"] == 1.0).all() and (a["barotr_fac2"] == 1.0).all()
    assert not a["rd_ws"].any() and not a["sn_u_ws"].any() and not a["sn_v_ws"].any()
    assert (a["uflux"][:, [0, -1]] == 0.0).all() and (a["vflux"][[0, -1], :] == 0.0).all()
    assert np.allclose(a["i_mass"] * a["mass_ws"], 1.0, rtol=1e-15)


@pytest.mark.parametrize("k4", [-1.0, 2.0e8])
def test_lateral_step_conserves_energy(k4):
    """With no source and no drag, the flux-form lateral step only moves
    mass-weighted energy between cells: sum(areaT * mass * E) is unchanged."""
    p = MI.random_case(40, 30, 7, 5, cdrag=0.0, gmcoeff=-1.0, kh_bg=500.0, k4=k4)
    q = p.copy()
    MO.step(q, 1)
    w = p.arrays["areaT"] * q.arrays["mass_ws"]
    d = w * (q.arrays["meke"] - p.arrays["meke"])
    assert np.abs(d).max() > 0.0
    assert abs(d.sum()) <= 1e-12 * np.abs(d).sum()


def test_gates_follow_meke_step_ext():
    """kh < 0 and k4 < 0: no lateral step (uflux, vflux, del2 untouched) and one drag half at full weight."""
    p = MI.random_case(20, 14, 5, 9, kh_bg=-1.0, k4=-1.0, **MI.all_terms())
    q = p.copy()
    MO.step(q, 1)
    for k in ("uflux", "vflux", "del2"):
        np.testing.assert_array_equal(q.arrays[k], p.arrays[k])
    # with the lateral step on, the fluxes are rewritten
    r = MI.random_case(20, 14, 5, 9, kh_bg=100.0, **MI.all_terms())
    s = r.copy()
    MO.step(s, 1)
    assert not np.array_equal(s.arrays["uflux"], r.arrays["uflux"])


def test_biharmonic_leaves_its_tendency_in_del2():
    p = MI.random_case(24, 18, 6, 11, k4=5.0e8, kh_bg=-1.0)
    q = p.copy()
    MO.step(q, 1)
    t = q.arrays["del2"]
    assert np.abs(t).max() > 0.0
    w = p.arrays["areaT"] * q.arrays["mass_ws"]
    assert abs((w * t).sum()) <= 1e-12 * np.abs(w * t).sum()


def test_golden_fixtures_present():
    assert len(GOLDEN) >= 4, "MEKE golden fixtures missing: run tests/golden/make_meke_golden.py on a GPU"


def _problem(z) -> MI.MekeProblem:
    nx, ny, nz = (int(z[k]) for k in ("nx", "ny", "nz"))
    arrays = {k[3:]: z[k].copy() for k in z.files if k.startswith("in_")}
    config = {k[4:]: float(z[k]) for k in z.files if k.startswith("cfg_")}
    return MI.MekeProblem(str(z["name"]), nx, ny, nz, arrays, config)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(g)[:-4] for g in GOLDEN])
def test_oracle_matches_reference_cuda(path):
    z = np.load(path)
    p = _problem(z)
    for s in range(int(z["nsteps"])):
        MO.step(p, 1)
        for k in MI.OUTPUTS:
            key = f"ref_step{s + 1}_{k}"
            if key in z.files:
                assert np.array_equal(p.arrays[k], z[key]), f"{k} after step {s + 1}"
