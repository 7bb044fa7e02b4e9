"""The allocation-free step, through the C-ABI.

`redi_b200_opt_launch_noalloc` is for callers that cannot allocate device
memory while they step the model (a cudaMalloc/cudaFree can stall the whole
device and is not allowed during stream capture; some host models own all
device memory through their own pool). It must give exactly the results of the
regular reference-compatible launcher `redi_opt_launch`, call after call, while
taking its scratch from a fixed array inside the library.
"""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU-only container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from more_benchmarks_dc_ocean_b200 import build, inputs  # noqa: E402


def _lib():
    build.build()
    from more_benchmarks_dc_ocean_b200 import ocean_redi as R

    L = R.lib()
    L.redi_b200_opt_launch_noalloc.restype = C.c_int
    return R, L


def _state(p):
    dev = "cuda"
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev, torch.float64)  # noqa: E731
    nx, ny, ns = p.nx, p.ny, p.ns
    st = {"h": d(p.h), "T": d(p.tracers[0]), "S": d(p.tracers[1]), "wet_u": d(p.wet_u), "wet_v": d(p.wet_v),
          "ku_ext": d(p.khtr_u), "kv_ext": d(p.khtr_v), "dy_cu": d(p.dy_cu), "dx_cv": d(p.dx_cv),
          "idxCu": d(p.idxCu), "idyCv": d(p.idyCv), "areaT": d(p.areaT)}
    for side, (a, b) in (("u", (ny, nx + 1)), ("v", (ny + 1, nx))):
        st[side + "PoL"] = torch.zeros((ns, a, b), dtype=torch.float64, device=dev)
        st[side + "PoR"] = torch.zeros((ns, a, b), dtype=torch.float64, device=dev)
        st[side + "KoL"] = torch.ones((ns, a, b), dtype=torch.int32, device=dev)
        st[side + "KoR"] = torch.ones((ns, a, b), dtype=torch.int32, device=dev)
        st[side + "hEff"] = torch.zeros((ns - 1, a, b), dtype=torch.float64, device=dev)
    st["ku"] = torch.zeros_like(st["ku_ext"])
    st["kv"] = torch.zeros_like(st["kv_ext"])
    st["snap"] = torch.zeros_like(st["T"])
    return st


def _args(p, st):
    ci = lambda v: C.byref(C.c_int(int(v)))  # noqa: E731
    cd = lambda v: C.byref(C.c_double(float(v)))  # noqa: E731
    vp = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    e = p.eos
    ww, we, ws, wn = p.walls
    return [ci(p.nx), ci(p.ny), ci(p.nz), ci(p.ns), cd(p.dt), ci(p.nghost), ci(p.nx_phys), ci(p.ny_phys),
            ci(ww), ci(we), ci(ws), ci(wn), cd(e.rho0), cd(e.T_ref), cd(e.S_ref), cd(e.alpha_T), cd(e.beta_S),
            vp(st["h"]), vp(st["T"]), vp(st["S"]), vp(st["wet_u"]), vp(st["wet_v"]),
            vp(st["uPoL"]), vp(st["uPoR"]), vp(st["uKoL"]), vp(st["uKoR"]), vp(st["uhEff"]),
            vp(st["vPoL"]), vp(st["vPoR"]), vp(st["vKoL"]), vp(st["vKoR"]), vp(st["vhEff"]),
            vp(st["ku_ext"]), vp(st["kv_ext"]), vp(st["ku"]), vp(st["kv"]),
            vp(st["dy_cu"]), vp(st["dx_cv"]), vp(st["idxCu"]), vp(st["idyCv"]), vp(st["areaT"]), vp(st["snap"])]


OUTPUTS = ("T", "S", "uPoL", "uPoR", "uKoL", "uKoR", "uhEff", "vPoL", "vPoR", "vKoL", "vKoR", "vhEff", "ku", "kv")


def test_noalloc_step_matches_regular_launcher_twice():
    """Two consecutive calls: every output equals the regular launcher's, bit for bit
    (the bar of the FP64 parity tests: both run the same FP64 kernels)."""
    R, L = _lib()
    p = inputs.make_problem(44, 36, 15, n_seamounts=4, land_fraction=0.2, seed=404)
    ref, got = _state(p), _state(p)
    stream = torch.cuda.current_stream()
    for call in range(2):
        L.redi_opt_launch(*_args(p, ref))
        rc = L.redi_b200_opt_launch_noalloc(*_args(p, got), C.c_void_p(stream.cuda_stream))
        assert rc == R.OK, R.last_error()
        torch.cuda.synchronize()
        for k in OUTPUTS:
            assert torch.equal(got[k], ref[k]), f"call {call + 1}: {k} differs"
        assert not torch.equal(got["T"], torch.from_numpy(p.tracers[0]).cuda()), "the step did nothing"


def test_noalloc_rejects_domains_beyond_its_scratch():
    """A domain whose scratch exceeds the fixed array is refused, untouched, with the limit in the message."""
    R, L = _lib()
    p = inputs.make_problem(150, 120, 40, n_seamounts=3, seed=5)
    st = _state(p)
    before = st["T"].clone()
    rc = L.redi_b200_opt_launch_noalloc(*_args(p, st), None)
    assert rc == R.E_UNSUPPORTED
    msg = R.last_error()
    assert "limited to 67108608 bytes" in msg, msg
    torch.cuda.synchronize()
    assert torch.equal(st["T"], before)


def test_noalloc_allocates_nothing_after_the_first_call():
    """After the first call on the device, further calls leave the device's free memory unchanged:
    no cudaMalloc, and no allocator cache growing behind the caller's back."""
    R, L = _lib()
    p = inputs.make_problem(44, 36, 15, n_seamounts=4, land_fraction=0.2, seed=405)
    st = _state(p)
    stream = torch.cuda.current_stream()
    assert L.redi_b200_opt_launch_noalloc(*_args(p, st), C.c_void_p(stream.cuda_stream)) == R.OK, R.last_error()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        assert L.redi_b200_opt_launch_noalloc(*_args(p, st), C.c_void_p(stream.cuda_stream)) == R.OK
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


def _need_bytes(nx, ny, nz):
    """The scratch the entry point asks for (the formula of csrc/redi_noalloc.cu)."""
    r = lambda b: (b + 255) & ~255  # noqa: E731
    ncol = nx * ny
    need_a = r(ncol * (nz + 1) * 32) + r(ncol * (nz + 1) * 8)
    need_b = (r(2 * ncol * (nz + 1) * 8) + r(2 * ncol * nz * 32) + r(2 * (2 * nz + 1) * (nx + 1) * ny * 8)
              + r(2 * (2 * nz + 1) * nx * (ny + 1) * 8))
    dry = r((nx + 1) * ny + nx * (ny + 1))  # the sweep's dry-face record, behind both phases
    return max(need_a, need_b) + dry


def test_noalloc_near_its_limit_at_75_layers():
    """The largest square domain that fits at nz = 75 (about 5 800 columns): every output equals
    redi_opt_launch's, bit for bit, on two calls in a row."""
    R, L = _lib()
    limit = (64 << 20) - 256
    n = max(k for k in range(40, 120) if _need_bytes(k + 4, k + 4, 75) <= limit)
    assert _need_bytes(n + 4, n + 4, 75) > 0.9 * limit
    p = inputs.make_problem(n, n, 75, n_seamounts=4, land_fraction=0.2, seed=406)
    ref, got = _state(p), _state(p)
    stream = torch.cuda.current_stream()
    for call in range(2):
        L.redi_opt_launch(*_args(p, ref))
        rc = L.redi_b200_opt_launch_noalloc(*_args(p, got), C.c_void_p(stream.cuda_stream))
        assert rc == R.OK, R.last_error()
        torch.cuda.synchronize()
        for k in OUTPUTS:
            assert torch.equal(got[k], ref[k]), f"call {call + 1}: {k} differs"
