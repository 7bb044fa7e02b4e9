"""The ALE remap step on the GPU (include/ale_b200.h) against the reference's own
CUDA and the oracle.

Bar: 0 ulp on every array the step writes, after every step. The fixtures hold
the outputs of the reference's `ale_remap_cuda` (ale_remap/ale_kernel.cu, FMA
contraction off); what its launchers do not implement (PCM, PLM, passive
tracers, the KE-conserving rescale, absent tracer slots or face velocities) is
checked against the CPU oracle restatement of ale_remap_step
(ale_remap/ale_remap.F90:76-188).
"""

import ctypes as C
import glob
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU-only container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from more_benchmarks_dc_ocean_b200 import ale_inputs as AI  # noqa: E402
from oracle import ale_oracle as AO  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "ale_*.npz")))


@pytest.fixture(scope="module")
def A(redi_lib):
    from more_benchmarks_dc_ocean_b200 import ale_remap

    return ale_remap


def _compare(got, want, what):
    for k in want:
        a, b = got[k], want[k]
        assert np.array_equal(a, b), f"{what}: {k} differs in {np.count_nonzero(a != b)} of {a.size} (max {np.abs(a - b).max():.3e})"


def _against_oracle(A, p, nsteps=2):
    d = A.to_device(p)
    q = p.copy()
    for s in range(nsteps):
        A.step_problem(p, d, 1)
        AO.step(q, 1)
        torch.cuda.synchronize()
        _compare(A.host_arrays(d), q.arrays(), f"{p.name} step {s + 1}")


def _fixture(path):
    z = np.load(path)
    g = lambda k: z["in_" + k].copy()  # noqa: E731
    p = AI.AleProblem(str(z["name"]), int(z["nx"]), int(z["ny"]), int(z["nz"]), g("h_layer"),
                      [g("tracer0"), g("tracer1")], g("u"), g("v"), g("mass_budget"), g("heat_budget"),
                      g("salt_budget"), g("bt_eta"), g("bt_H_ref"), g("dsig"))
    return z, p


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(g)[:-4] for g in GOLDEN])
def test_matches_reference_cuda(A, path):
    z, p = _fixture(path)
    d = A.to_device(p)
    for s in range(int(z["nsteps"])):
        A.step_problem(p, d, 1)
        torch.cuda.synchronize()
        got = A.host_arrays(d)
        want = {k: z[f"ref_step{s + 1}_{k}"] for k in got if f"ref_step{s + 1}_{k}" in z.files}
        _compare(got, want, f"{p.name} step {s + 1}")


@pytest.mark.parametrize("method", [AI.REMAP_PCM, AI.REMAP_PLM, AI.REMAP_PPM, 0, 7])
@pytest.mark.parametrize("conserve_ke", [False, True])
def test_methods_and_ke_rescale_match_oracle(A, method, conserve_ke):
    p = AI.random_case(23, 19, 14, 500 + method, method=method, conserve_ke=conserve_ke, n_passive=2,
                       name=f"m{method}_ke{int(conserve_ke)}")
    _against_oracle(A, p)


@pytest.mark.parametrize("nz", [1, 2, 3, 31, 32, 33, 64, 65, 128])
def test_column_capacities_match_oracle(A, nz):
    p = AI.random_case(11, 9, nz, 600 + nz, n_passive=1, zero_targets=min(3, max(0, nz - 3)), name=f"nz{nz}")
    _against_oracle(A, p)


@pytest.mark.parametrize("shape", [(1, 7, 6), (7, 1, 6), (1, 1, 4), (2, 3, 5)])
def test_small_shapes_match_oracle(A, shape):
    p = AI.random_case(*shape, 700 + sum(shape), n_passive=1, conserve_ke=True, name=f"shape{shape}")
    _against_oracle(A, p)


def test_many_tracers_absent_slots_no_faces(A):
    """11 slots (two launches of tracers), two of them unallocated, no face velocities."""
    p = AI.random_case(19, 15, 10, 801, n_passive=9, faces=False, name="many")
    p.tracers[4] = None
    p.tracers[7] = None
    p.idx_temperature, p.idx_salinity = 2, 5
    _against_oracle(A, p)


def test_reference_benchmark_size_matches_oracle(A):
    p = AI.reference_ic()
    _against_oracle(A, p, nsteps=1)


def test_reference_signature_exports(A):
    """ale_remap_cuda (both forms) and ale_remap_opt give the step's results (PPM, T and S)."""
    for how in (0, 1, "opt"):
        p = AI.random_case(25, 18, 12, 901, n_passive=0, name=f"export{how}")
        d = A.to_device(p)
        T, S = d["tracers"]
        g = d
        if how == "opt":
            A.ale_remap_opt(p.nx, p.ny, p.nz, g["h_layer"], g["h_old"], g["target_h"], T, S, g["u"], g["v"],
                            g["mass_budget"], g["heat_budget"], g["salt_budget"], g["bt_eta"], g["bt_H_ref"],
                            g["dsig"])
        else:
            A.ale_remap_cuda(p.nx, p.ny, p.nz, 3, how, g["h_layer"], g["h_old"], g["target_h"], g["total_h"],
                             g["h_ref"], T, S, g["u"], g["v"], g["mass_budget"], g["heat_budget"],
                             g["salt_budget"], g["bt_eta"], g["bt_H_ref"], g["dsig"])
        A.lib().cuda_sync()
        q = p.copy()
        AO.step(q, 1)
        want = q.arrays()
        if how == "opt":  # the reference's optimized launcher has no total_h / h_ref outputs
            want = {k: v for k, v in want.items() if k not in ("total_h", "h_ref")}
        _compare(A.host_arrays(d), want, f"export {how}")


def test_python_mirror_of_ale_remap_step(A):
    p = AI.random_case(27, 21, 13, 1001, n_passive=1, conserve_ke=True)
    d = A.to_device(p)
    grid = A.AleGrid(p.nx, p.ny)
    vc = A.OceanVcoord(p.nz, d["dsig"], d["target_h"], d["h_old"], d["total_h"], d["h_ref"],
                       remap_method=p.method, remap_vel_conserve_ke=True)
    ms = A.AleState(p.nz, d["h_layer"], d["tracers"], d["u"], d["v"], d["mass_budget"], d["heat_budget"],
                    d["salt_budget"], idx_temperature=p.idx_temperature + 1, idx_salinity=p.idx_salinity + 1)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        A.ale_remap_step(grid, vc, ms, d["bt_eta"], d["bt_H_ref"])
    s.synchronize()
    q = p.copy()
    AO.step(q, 1)
    _compare(A.host_arrays(d), q.arrays(), "ale_remap_step")
    with pytest.raises(A.AleError):
        A.ale_remap_step(grid, A.OceanVcoord(p.nz, d["dsig"], d["target_h"], d["h_old"], d["total_h"], d["h_ref"],
                                             coord_type=5), ms, d["bt_eta"], d["bt_H_ref"])


def test_launches_counted(A, redi_lib):
    L = redi_lib.lib()
    L.redi_b200_launch_count.restype = C.c_ulonglong
    before = [L.redi_b200_launch_count(k) for k in (13, 14)]
    p = AI.random_case(12, 10, 6, 4, n_passive=8)  # 10 tracers: two tracer launches
    d = A.to_device(p)
    A.step_problem(p, d, 2)
    torch.cuda.synchronize()
    after = [L.redi_b200_launch_count(k) for k in (13, 14)]
    assert [b - a for a, b in zip(before, after)] == [4, 2]
