"""The MEKE step on the GPU (include/meke_b200.h) against the oracle and the
reference's own CUDA.

Bar: 0 ulp on every array the step writes, after every step. The fixtures hold
the outputs of the reference's `meke_cuda_launch` (meke/meke_kernel.cu, FMA
contraction off); the branches its launchers do not implement (kh < 0, k4 >= 0)
and the shapes they cannot launch (ny == 1) are checked against the CPU oracle
restatement of meke_step_ext (meke/meke.F90:60-131).
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

from more_benchmarks_dc_ocean_b200 import meke_inputs as MI  # noqa: E402
from oracle import meke_oracle as MO  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "meke_*.npz")))


@pytest.fixture(scope="module")
def M(redi_lib):
    from more_benchmarks_dc_ocean_b200 import ocean_meke

    return ocean_meke


class _View:
    def __init__(self, ptr, shape):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": "<f8", "data": (ptr, False), "version": 3}


def _device_view(ptr, shape):
    return torch.as_tensor(_View(ptr, shape), device="cuda")


def _host(d):
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in d.items()}


def _compare(got, want, keys, what):
    for k in keys:
        a, b = got[k], want[k]
        assert np.array_equal(a, b), f"{what}: {k} differs in {np.count_nonzero(a != b)} of {a.size} (max {np.abs(a - b).max():.3e})"


def _against_oracle(M, p, nsteps=3, keys=MI.OUTPUTS):
    d = M.to_device(p)
    h = None
    q = p.copy()
    try:
        for s in range(nsteps):
            h = M.step_problem(p, d, 1, handle=h)
            MO.step(q, 1)
            _compare(_host(d), q.arrays, keys, f"{p.name} step {s + 1}")
    finally:
        if h:
            M.destroy_handle(h)


def _fixture(path):
    z = np.load(path)
    arrays = {k[3:]: z[k].copy() for k in z.files if k.startswith("in_")}
    config = {k[4:]: float(z[k]) for k in z.files if k.startswith("cfg_")}
    return z, MI.MekeProblem(str(z["name"]), int(z["nx"]), int(z["ny"]), int(z["nz"]), arrays, config)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(g)[:-4] for g in GOLDEN])
def test_matches_reference_cuda(M, path):
    z, p = _fixture(path)
    d = M.to_device(p)
    h = None
    try:
        for s in range(int(z["nsteps"])):
            h = M.step_problem(p, d, 1, handle=h)
            got = _host(d)
            want = {k: z[f"ref_step{s + 1}_{k}"] for k in MI.OUTPUTS if f"ref_step{s + 1}_{k}" in z.files}
            _compare(got, want, want.keys(), f"{p.name} step {s + 1}")
    finally:
        if h:
            M.destroy_handle(h)


CASES = {
    "no_lateral": dict(kh_bg=-1.0, k4=-1.0),
    "biharmonic_only": dict(kh_bg=-1.0, k4=4.0e8),
    "biharmonic_and_laplacian": dict(kh_bg=250.0, k4=4.0e8, khmeke_fac=0.4),
    "biharmonic_cfl_clip": dict(kh_bg=100.0, k4=1.0e13),
    "all_terms": MI.all_terms(),
    "gm_off_frcoeff_on": dict(gmcoeff=-1.0, frcoeff=0.8, cdrag=0.0),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_branches_match_oracle(M, case):
    p = MI.random_case(33, 27, 13, 300 + sorted(CASES).index(case), name=case, **CASES[case])
    _against_oracle(M, p)


@pytest.mark.parametrize("shape", [(1, 9, 4), (9, 1, 4), (1, 1, 2), (2, 2, 1), (37, 5, 0), (64, 3, 8), (5, 7, 16)])
def test_edge_shapes_match_oracle(M, shape):
    nx, ny, nz = shape
    p = MI.random_case(nx, ny, nz, 17 + nx + ny, name=f"shape_{nx}x{ny}x{nz}", **MI.all_terms(k4=1.0e8))
    _against_oracle(M, p, nsteps=2)


def test_reference_benchmark_size_matches_oracle(M):
    """The reference's benchmark (473 x 297 points, 3 ghosts, 30 layers), 10 steps."""
    p = MI.reference_ic()
    d = M.to_device(p)
    h = M.step_problem(p, d, 10)
    got = _host(d)
    M.destroy_handle(h)
    q = p.copy()
    MO.step(q, 10)
    _compare(got, q.arrays, MI.OUTPUTS, "reference IC, 10 steps")


def test_python_mirror_of_meke_step_ext(M):
    p = MI.random_case(40, 31, 9, 77, **MI.all_terms(k4=2.0e8))
    d = M.to_device(p)
    m = M.OceanMeke(enable=True)
    m.nx_total, m.ny_total, m.nz_ml = p.nx, p.ny, p.nz
    m.is_init = True
    for n in M.OceanMeke.ARRAYS:
        m.arrays[n] = d[n]
    c = p.config
    for attr, key in (("gmcoeff", "gmcoeff"), ("frcoeff", "frcoeff"), ("bgsrc", "bgsrc"), ("damping", "damping"),
                      ("kh", "kh_bg"), ("k4", "k4"), ("khmeke_fac", "khmeke_fac"), ("khcoeff", "khcoeff"),
                      ("cd_scale", "cd_scale"), ("cb", "cb"), ("ct", "ct"), ("min_gamma2", "min_gamma2"),
                      ("uscale", "uscale"), ("dtscale", "dtscale"), ("cdrag", "cdrag"),
                      ("alpha_deform", "a_deform"), ("alpha_rhines", "a_rhines"), ("alpha_eady", "a_eady"),
                      ("alpha_frict", "a_frict"), ("alpha_grid", "a_grid"), ("visc_coeff_ku", "visc_coeff_ku")):
        setattr(m, attr, c[key])
    m.backscatter = bool(c["backscatter"])
    metrics = M.MekeMetrics(*(d[k] for k in ("areaT", "iareaT", "idxT", "idyT", "dy_cu", "dx_cv", "idxCu", "idyCv")))
    ms = M.MekeLayers(p.nz, d["h_layer"], d["rho_layer"])
    gm = M.OceanGM(d["gm_src"], rho0=c["rho0"])
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        for _ in range(2):
            M.meke_step_ext(p.nx, p.ny, p.nz, m, metrics, gm, ms, c["dt"], d["ke_diss_ext"])
    s.synchronize()
    m.destroy()
    q = p.copy()
    MO.step(q, 2)
    _compare(_host(d), q.arrays, MI.OUTPUTS, "meke_step_ext")


def _compat_run(M, p, how, nsteps=2):
    d = M.to_device(p)
    a = M.make_args(p.nx, p.ny, p.nz, d, p.config)
    scratch = torch.zeros(p.ny, p.nx, dtype=torch.float64, device="cuda")
    for _ in range(nsteps):
        if how == "opt":
            M.meke_opt_launch(a, scratch)
        else:
            M.meke_cuda_launch(a, how)
    M.meke_cuda_graph_reset()
    return _host(d), scratch.cpu().numpy()


@pytest.mark.parametrize("how", [0, 1, 2, "opt"])
def test_reference_signature_exports(M, how):
    """meke_cuda_launch modes 0/1/2 and meke_opt_launch give the step's results;
    meke_opt_launch leaves the post-drag energy in the caller's scratch."""
    p = MI.random_case(45, 38, 10, 91, **MI.all_terms(k4=3.0e8))
    got, scratch = _compat_run(M, p, how)
    q = p.copy()
    MO.step(q, 2)
    keys = [k for k in MI.OUTPUTS if k != "del2"]  # MekeArgs has no del2 slot
    _compare(got, q.arrays, keys, f"export {how}")
    if how == "opt":
        # the caller's scratch holds the post-drag energy of the last step, as the handle's own scratch does
        d2 = M.to_device(p)
        h = M.step_problem(p, d2, 2)
        torch.cuda.synchronize()
        e1 = _device_view(M.lib().meke_b200_scratch_energy(h), (p.ny, p.nx)).cpu().numpy()
        M.destroy_handle(h)
        assert np.array_equal(scratch, e1)
    assert not np.isnan(scratch).any()


def test_graph_mode_recaptures_when_arguments_change(M):
    p1 = MI.random_case(20, 15, 6, 5, **MI.all_terms())
    p2 = MI.random_case(20, 15, 6, 6, **MI.all_terms(kh_bg=50.0))
    d1, d2 = M.to_device(p1), M.to_device(p2)
    a1 = M.make_args(p1.nx, p1.ny, p1.nz, d1, p1.config)
    a2 = M.make_args(p2.nx, p2.ny, p2.nz, d2, p2.config)
    M.meke_cuda_launch(a1, 2)
    M.meke_cuda_launch(a2, 2)
    M.meke_cuda_launch(a1, 2)
    M.meke_cuda_graph_reset()
    q1, q2 = p1.copy(), p2.copy()
    MO.step(q1, 2)
    MO.step(q2, 1)
    keys = [k for k in MI.OUTPUTS if k != "del2"]
    _compare(_host(d1), q1.arrays, keys, "graph, domain 1")
    _compare(_host(d2), q2.arrays, keys, "graph, domain 2")


def test_fluxes_optional(M):
    """uflux / vflux may be NULL: everything else is unchanged."""
    p = MI.random_case(25, 19, 7, 8, **MI.all_terms())
    d = M.to_device(p)
    d_no = {k: v for k, v in M.to_device(p).items() if k not in ("uflux", "vflux")}
    h1 = M.step_problem(p, d, 1)
    h2 = M.step_problem(p, d_no, 1)
    M.destroy_handle(h1)
    M.destroy_handle(h2)
    a, b = _host(d), _host(d_no)
    _compare(b, a, [k for k in MI.OUTPUTS if k not in ("uflux", "vflux")], "without fluxes")


def test_launches_counted(M, redi_lib):
    L = redi_lib.lib()
    L.redi_b200_launch_count.restype = C.c_ulonglong
    before = [L.redi_b200_launch_count(k) for k in (10, 11, 12)]
    p = MI.random_case(16, 12, 5, 4, k4=1.0e8)
    d = M.to_device(p)
    h = M.step_problem(p, d, 3)
    M.destroy_handle(h)
    torch.cuda.synchronize()
    after = [L.redi_b200_launch_count(k) for k in (10, 11, 12)]
    assert [b - a for a, b in zip(before, after)] == [3, 3, 3]
