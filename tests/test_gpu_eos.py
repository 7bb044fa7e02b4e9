"""The non-linear equations of state on the GPU, against the CPU oracle.

The column state evaluates the reference's point EOS (redi/ocean_eos.F90:450-546)
at every interface; with WRIGHT_97 or ROQUET_SPV the density and its
derivatives depend on the interface pressure. The device code and the oracle
are written independently from the reference; both are compiled without FMA
contraction, so the bar is 0 ulp: at single points (redi_b200_eos_points), and
through whole steps (coefficients and tracers), alone and inside the
multi-domain batch.
"""

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU-only container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from more_benchmarks_dc_ocean_b200 import inputs  # noqa: E402
from oracle import oracle as O  # noqa: E402

VARIANTS = [1, 2, 4]


def _samples(n=4096, seed=7):
    r = np.random.default_rng(seed)
    T = r.uniform(-2.0, 32.0, n)
    S = r.uniform(0.0, 40.0, n)
    p = r.uniform(0.0, 6.0e7, n)
    S[:8] = 0.0  # fresh water: the floor under the CT polynomial's square root
    p[8:16] = 0.0
    return T, S, p


@pytest.mark.parametrize("variant", VARIANTS)
def test_eos_points_match_oracle(redi_lib, oracle_lib, variant):
    R = redi_lib
    T, S, p = _samples()
    e = R.OceanEos(alpha_T=2e-4, variant=variant)
    d = lambda a: torch.from_numpy(a).cuda()  # noqa: E731
    rho, dT, dS = (t.cpu().numpy() for t in R.eos_points(e, d(T), d(S), d(p)))
    torch.cuda.synchronize()
    oe = inputs.Eos(alpha_T=2e-4, variant=variant)
    ref = np.array([O.eos_point(oe, a, b, c) for a, b, c in zip(T, S, p)])
    for name, got, want in (("rho", rho, ref[:, 0]), ("dsv_dt", dT, ref[:, 1]), ("dsv_ds", dS, ref[:, 2])):
        assert np.array_equal(got, want), f"variant {variant} {name}: {np.count_nonzero(got != want)} differ"


@pytest.mark.parametrize("variant,name", [(1, "linear"), (2, "wright")])
def test_eos_points_match_reference_cuda(redi_lib, variant, name):
    """dSV/dT and dSV/dS against the reference's own CUDA eos_specvol_derivs
    (epbl/epbl_kernel.cu:112-137 and kappa_shear/ks_kernel.cu:108-134, fixture
    tests/golden/eos_specvol_ref.npz), 0 ulp."""
    R = redi_lib
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "eos_specvol_ref.npz"))
    e = R.OceanEos(variant=variant, rho0=float(z["cfg_rho0"]), alpha_T=float(z["cfg_alpha_T"]),
                   beta_S=float(z["cfg_beta_S"]))
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    _, dT, dS = R.eos_points(e, d(z["T"]), d(z["S"]), d(z["p"]))
    torch.cuda.synchronize()
    for dname, got in (("dsv_dt", dT.cpu().numpy()), ("dsv_ds", dS.cpu().numpy())):
        for copy in ("epbl", "ks"):
            want = z[f"{copy}_{name}_{dname}"]
            assert np.array_equal(got, want), f"{copy} {dname}: {np.count_nonzero(got != want)} differ"


def _problem(variant, seed=31):
    p = inputs.make_problem(24, 20, 12, n_seamounts=3, land_fraction=0.2, seed=seed)
    p.eos = inputs.Eos(rho0=1035.0, variant=variant)
    return p


@pytest.mark.parametrize("variant", [2, 4])
def test_step_with_nonlinear_eos_matches_oracle(redi_lib, oracle_lib, variant):
    """Two full steps: every coefficient and every tracer value, 0 ulp."""
    R = redi_lib
    p = _problem(variant)
    dp = R.to_device(p)
    redi = R.make_redi(dp)
    R.step(dp, redi, 2)
    torch.cuda.synchronize()
    got = {k: v.cpu().numpy() for k, v in redi.coeffs().items()}
    trs = [t.cpu().numpy() for t in dp.ms.tracers]
    redi.destroy()
    q = p.copy()
    c = O.step(q, 2)
    for k in ("uPoL", "uPoR", "uKoL", "uKoR", "uhEff", "vPoL", "vPoR", "vKoL", "vKoR", "vhEff"):
        assert np.array_equal(got[k], c[k]), f"variant {variant} {k}"
    for n, (a, b) in enumerate(zip(trs, q.tracers)):
        assert np.array_equal(a, b), f"variant {variant} tracer {n}"
    # the non-linear EOS changes the neutral surfaces: not the linear answer
    lin = _problem(1)
    O.step(lin, 2)
    assert not np.array_equal(q.tracers[0], lin.tracers[0])


def test_mixed_precision_with_wright_eos(redi_lib, oracle_lib):
    R = redi_lib
    p = _problem(2)
    dp = R.to_device(p)
    redi = R.make_redi(dp, R.MIXED)
    R.step(dp, redi, 1)
    torch.cuda.synchronize()
    trs = [t.cpu().numpy() for t in dp.ms.tracers]
    redi.destroy()
    q = p.copy()
    O.step(q, 1)
    for n, (a, b) in enumerate(zip(trs, q.tracers)):
        err = float(np.abs(a - b).max()) / float(np.abs(b).max())
        assert err <= 1e-7, (n, err)


def test_batch_with_mixed_eos_variants(redi_lib, oracle_lib):
    """One persistent launch over domains that each use a different EOS."""
    R = redi_lib
    ps = [_problem(v, seed=40 + v) for v in VARIANTS]
    dps = [R.to_device(p) for p in ps]
    b = R.RediBatch(dps)
    b.step(2)
    torch.cuda.synchronize()
    assert b.status()["status"] == 0
    b.destroy()
    for p, dp in zip(ps, dps):
        q = p.copy()
        O.step(q, 2)
        for n, (t, r) in enumerate(zip(dp.ms.tracers, q.tracers)):
            assert np.array_equal(t.cpu().numpy(), r), (p.eos.variant, n)


def test_eos_variant_codes_checked(redi_lib):
    R = redi_lib
    p = _problem(1)
    dp = R.to_device(p)
    redi = R.make_redi(dp)
    for code, err in ((3, R.E_UNSUPPORTED), (7, R.E_ARG)):
        dp.eos.variant = code
        with pytest.raises(R.RediError) as ex:
            R.redi_calc_coeffs(dp.grid, dp.metrics, dp.eos, redi, dp.ms)
        assert ex.value.code == err
    redi.destroy()
