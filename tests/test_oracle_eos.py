"""The oracle's point equation of state: the non-linear branches of redi/ocean_eos.F90.

The reference's Redi CUDA implements the linear branch only, and its Fortran
cannot be compiled here. The WRIGHT_97 specific-volume derivatives are pinned
bit for bit against the reference's own CUDA transcriptions of
eos_specvol_derivs in two other models (epbl/epbl_kernel.cu:112-137,
kappa_shear/ks_kernel.cu:108-134), run on a B200 by
tests/golden/make_eos_golden.py (fixture eos_specvol_ref.npz). The WRIGHT_97
density and the ROQUET_SPV branch exist in no compiled form of the reference;
they are pinned by what the reference itself uses to check them
(ocean_eos.F90:300-306, 516-525): the specific-volume derivatives must equal
finite differences of the specific volume, densities must be those of seawater,
and the two independent fits (Wright 1997, Roquet 2015) must agree over the
oceanic range.
"""

import os

import numpy as np
import pytest

from more_benchmarks_dc_ocean_b200.inputs import Eos
from oracle import oracle as O

WRIGHT, ROQUET = 2, 4
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "eos_specvol_ref.npz")
POINTS = [(T, S, p) for T in (-1.5, 2.0, 10.0, 18.0, 29.0) for S in (30.0, 34.7, 35.0, 37.5)
          for p in (0.0, 1.0e7, 4.0e7)]


def _sv(variant, T, S, p):
    if variant == ROQUET:
        return O.roquet_sv(T, S, p)
    rho, _, _ = O.eos_point(Eos(variant=variant), T, S, p)
    return 1.0 / rho


@pytest.mark.parametrize("variant", [WRIGHT, ROQUET])
def test_derivatives_match_finite_differences(oracle_lib, variant):
    """dSV/dT and dSV/dS against centred differences of SV (second order, h = 1e-3)."""
    h = 1.0e-3
    for T, S, p in POINTS:
        _, dT, dS = O.eos_point(Eos(variant=variant), T, S, p)
        fdT = (_sv(variant, T + h, S, p) - _sv(variant, T - h, S, p)) / (2 * h)
        fdS = (_sv(variant, T, S + h, p) - _sv(variant, T, S - h, p)) / (2 * h)
        assert abs(dT - fdT) <= 1e-5 * abs(dT) + 1e-14, (variant, T, S, p, dT, fdT)
        assert abs(dS - fdS) <= 1e-5 * abs(dS) + 1e-14, (variant, T, S, p, dS, fdS)


@pytest.mark.parametrize("variant", [WRIGHT, ROQUET])
def test_seawater_densities(oracle_lib, variant):
    rho, dT, dS = O.eos_point(Eos(variant=variant), 10.0, 35.0, 0.0)
    assert 1026.5 < rho < 1027.5, rho
    assert dT > 0 and dS < 0  # warm water expands, salt contracts
    rho_deep, _, _ = O.eos_point(Eos(variant=variant), 2.0, 34.7, 4.0e7)  # about 4000 m
    assert 1044.0 < rho_deep < 1047.0, rho_deep


def test_wright_and_roquet_agree(oracle_lib):
    """Two independent fits of seawater: densities within 3e-5, derivatives within 3 %."""
    for T, S, p in POINTS:
        if S < 33.0 and T > 25.0:
            continue
        rw, tw, sw = O.eos_point(Eos(variant=WRIGHT), T, S, p)
        rr, tr, sr = O.eos_point(Eos(variant=ROQUET), T, S, p)
        assert abs(rw - rr) <= 3e-5 * rr, (T, S, p, rw, rr)
        assert abs(tw - tr) <= 0.03 * abs(tr) + 2e-9, (T, S, p, tw, tr)
        assert abs(sw - sr) <= 0.03 * abs(sr), (T, S, p, sw, sr)


def test_linear_variant_codes(oracle_lib):
    """0 (a zero-initialised handle) and 1 (EOS_VARIANT_LINEAR) are the linear branch."""
    e1, e0 = Eos(variant=1, alpha_T=2e-4), Eos(variant=0, alpha_T=2e-4)
    for T, S, p in POINTS[:6]:
        a, b = O.eos_point(e1, T, S, p), O.eos_point(e0, T, S, p)
        assert a == b
        assert a[0] == 1035.0 + 7.6e-4 * (S - 35.0) - 2e-4 * (T - 10.0)


@pytest.mark.parametrize("copy", ["epbl", "ks"])
@pytest.mark.parametrize("variant,name", [(1, "linear"), (WRIGHT, "wright")])
def test_specvol_derivs_match_reference_cuda(oracle_lib, copy, variant, name):
    """dSV/dT and dSV/dS at 2318 points, 0 ulp against each reference CUDA copy."""
    z = np.load(GOLDEN)
    e = Eos(variant=variant, rho0=float(z["cfg_rho0"]), alpha_T=float(z["cfg_alpha_T"]),
            beta_S=float(z["cfg_beta_S"]))
    got = np.array([O.eos_point(e, a, b, c)[1:] for a, b, c in zip(z["T"], z["S"], z["p"])])
    for i, d in enumerate(("dsv_dt", "dsv_ds")):
        want = z[f"{copy}_{name}_{d}"]
        assert np.array_equal(got[:, i], want), f"{d}: {np.count_nonzero(got[:, i] != want)} of {want.size} differ"
