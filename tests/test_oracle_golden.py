"""The CPU oracle against golden vectors produced by the reference's own CUDA.

Each Redi fixture in tests/golden/*.npz (the meke_* and ale_* fixtures belong to
the MEKE and ALE remap steps, test_meke_cpu.py and test_ale_cpu.py, and the eos_*
fixture to the point EOS, test_oracle_eos.py) holds seeded
inputs and the outputs of the
reference launcher `redi_opt_launch` (redi/opt_kernel.cu, built from the
reference sources with FMA contraction off; see tests/golden/make_golden.py):
Phase-A coefficients after the last step and T, S after every step. The oracle
must reproduce them bit for bit.
"""

import glob
import os

import numpy as np
import pytest

from more_benchmarks_dc_ocean_b200.inputs import Eos, RediProblem

GOLDEN = sorted(g for g in glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz"))
                if not os.path.basename(g).startswith(("meke_", "ale_", "eos_")))


def _problem(z) -> RediProblem:
    e = z["eos"]
    return RediProblem(
        name="golden", nx_phys=int(z["nx_phys"]), ny_phys=int(z["ny_phys"]), nz=int(z["nz"]),
        nghost=int(z["nghost"]), dt=float(z["dt"]), eos=Eos(*map(float, e)), h=z["h"].copy(),
        tracers=[z["T0"].copy(), z["S0"].copy()], idx_temperature=0, idx_salinity=1,
        dy_cu=z["dy_cu"], dx_cv=z["dx_cv"], idxCu=z["idxCu"], idyCv=z["idyCv"], areaT=z["areaT"],
        wet_u=z["wet_u"], wet_v=z["wet_v"], khtr_u=z["khtr_u"], khtr_v=z["khtr_v"],
        walls=tuple(int(w) for w in z["walls"]))


def test_fixtures_present():
    assert len(GOLDEN) >= 5, "golden fixtures missing: run tests/golden/make_golden.py on a GPU"


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(g)[:-4] for g in GOLDEN])
def test_oracle_matches_reference_cuda(path, oracle_lib):
    z = np.load(path)
    p = _problem(z)
    c = oracle_lib.new_coeffs(p.nx, p.ny, p.nz)
    nsteps = int(z["nsteps"])
    for s in range(nsteps):
        oracle_lib.calc_coeffs(p, c)
        if s == nsteps - 1:
            for k in c:
                assert np.array_equal(c[k], z["ref_" + k]), k
        oracle_lib.apply_flux(p, c)
        assert np.array_equal(p.tracers[0], z[f"ref_step{s + 1}_T"]), f"T after step {s + 1}"
        assert np.array_equal(p.tracers[1], z[f"ref_step{s + 1}_S"]), f"S after step {s + 1}"
