"""ctypes front end of the CPU oracle (oracle/redi_oracle.cpp).

TEST INFRASTRUCTURE ONLY. Imported by tests/, by the smoke check and by
bench.py's CPU-baseline / reference arm, always as the checker or the timed CPU
baseline — never as the product path.

Arrays follow the reference's Fortran memory layout; numpy shapes are the
Fortran shapes reversed (see more_benchmarks_dc_ocean_b200/inputs.py).
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libredi_oracle.so")
_lock = threading.Lock()
_lib = None

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def build() -> str:
    """Compile the oracle shared library (make -C oracle)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    with _lock:
        if _lib is None:
            srcs = [os.path.join(_HERE, f) for f in ("redi_oracle.cpp", "redi_eos_oracle.h")]
            if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < max(map(os.path.getmtime, srcs)):
                build()
            L = C.CDLL(_LIB_PATH)
            L.redi_oracle_calc_coeffs.restype = None
            L.redi_oracle_eos_point.restype = None
            L.redi_oracle_eos_point.argtypes = [C.c_int] + [C.c_double] * 8 + [_dp] * 3
            L.redi_oracle_roquet_sv.restype = C.c_double
            L.redi_oracle_roquet_sv.argtypes = [C.c_double] * 3
            L.redi_oracle_apply_flux.restype = None
            L.redi_oracle_count_ops.restype = None
            L.redi_oracle_max_threads.restype = C.c_int
            _lib = L
    return _lib


def _d(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous, (a.dtype, a.flags)
    return a.ctypes.data_as(_dp)


def _i(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_ip)


def new_coeffs(nx: int, ny: int, nz: int) -> dict:
    """Coefficient slots as ocean_redi_init leaves them (ocean_redi.F90:493-502)."""
    ns = 2 * nz + 2
    c = {}
    for side, (a, b) in (("u", (ny, nx + 1)), ("v", (ny + 1, nx))):
        c[side + "PoL"] = np.zeros((ns, a, b))
        c[side + "PoR"] = np.zeros((ns, a, b))
        c[side + "KoL"] = np.ones((ns, a, b), dtype=np.int32)
        c[side + "KoR"] = np.ones((ns, a, b), dtype=np.int32)
        c[side + "hEff"] = np.zeros((ns - 1, a, b))
    return c


def calc_coeffs(p, coeffs: dict | None = None, nthreads: int = 0) -> dict:
    """redi_calc_coeffs (ocean_redi.F90:572-607) on problem ``p``."""
    c = coeffs if coeffs is not None else new_coeffs(p.nx, p.ny, p.nz)
    e = p.eos
    T = np.ascontiguousarray(p.tracers[p.idx_temperature])
    S = np.ascontiguousarray(p.tracers[p.idx_salinity])
    lib().redi_oracle_calc_coeffs(
        p.nx, p.ny, p.nz, p.ns, C.c_double(e.rho0), C.c_double(e.T_ref), C.c_double(e.S_ref),
        C.c_double(e.alpha_T), C.c_double(e.beta_S), _d(p.h), _d(T), _d(S), _d(p.wet_u), _d(p.wet_v),
        _d(c["uPoL"]), _d(c["uPoR"]), _i(c["uKoL"]), _i(c["uKoR"]), _d(c["uhEff"]),
        _d(c["vPoL"]), _d(c["vPoR"]), _i(c["vKoL"]), _i(c["vKoR"]), _d(c["vhEff"]), nthreads,
        int(getattr(e, "variant", 1)))
    return c


def eos_point(eos, T: float, S: float, p: float):
    """(rho, dSV/dT, dSV/dS) at one point, as redi_build_column combines the reference's
    eos_density_point and eos_specvol_derivs (ocean_eos.F90:450-546)."""
    out = [C.c_double() for _ in range(3)]
    lib().redi_oracle_eos_point(int(getattr(eos, "variant", 1)), eos.rho0, eos.T_ref, eos.S_ref, eos.alpha_T,
                                eos.beta_S, float(T), float(S), float(p), *[C.byref(o) for o in out])
    return tuple(o.value for o in out)


def roquet_sv(T: float, S: float, p: float) -> float:
    """Specific volume of the Roquet (2015) polynomial (roquet_spv_point's sv)."""
    return lib().redi_oracle_roquet_sv(float(T), float(S), float(p))


def apply_flux(p, coeffs: dict, tracers=None, nthreads: int = 0):
    """redi_apply_flux (ocean_redi.F90:927-1002): updates ``tracers`` (default p.tracers) in place."""
    trs = p.tracers if tracers is None else tracers
    for t in trs:
        assert t.shape == (p.nz, p.ny, p.nx) and t.flags.c_contiguous
    arr = (_dp * len(trs))(*[_d(t) for t in trs])
    ww, we, ws, wn = p.walls
    c = coeffs
    lib().redi_oracle_apply_flux(
        p.nx, p.ny, p.nz, p.ns, C.c_double(p.dt), p.nghost, p.nx_phys, p.ny_phys, ww, we, ws, wn,
        _d(p.khtr_u), _d(p.khtr_v), _d(p.dy_cu), _d(p.dx_cv), _d(p.idxCu), _d(p.idyCv), _d(p.areaT),
        _d(p.h), len(trs), arr,
        _d(c["uPoL"]), _d(c["uPoR"]), _i(c["uKoL"]), _i(c["uKoR"]), _d(c["uhEff"]),
        _d(c["vPoL"]), _d(c["vPoR"]), _i(c["vKoL"]), _i(c["vKoR"]), _d(c["vhEff"]), nthreads)
    return trs


def step(p, nsteps: int = 1, nthreads: int = 0, coeffs: dict | None = None):
    """``nsteps`` full Redi steps (Phase A then Phase B on every tracer), in place on p.tracers."""
    c = coeffs if coeffs is not None else new_coeffs(p.nx, p.ny, p.nz)
    for _ in range(nsteps):
        calc_coeffs(p, c, nthreads)
        apply_flux(p, c, None, nthreads)
    return c


def count_ops(p):
    """Exact FP64 op counts of one step: (phase_A, phase_B) dicts of add/mul/div/cmp/cvt."""
    c = new_coeffs(p.nx, p.ny, p.nz)
    trs = [t.copy() for t in p.tracers]
    arr = (_dp * len(trs))(*[_d(t) for t in trs])
    a = (C.c_uint64 * 5)()
    b = (C.c_uint64 * 5)()
    e = p.eos
    lib().redi_oracle_count_ops(
        p.nx, p.ny, p.nz, p.ns, C.c_double(e.rho0), C.c_double(e.T_ref), C.c_double(e.S_ref),
        C.c_double(e.alpha_T), C.c_double(e.beta_S), C.c_double(p.dt), p.nghost, p.nx_phys, p.ny_phys,
        _d(p.h), len(trs), arr, _d(p.wet_u), _d(p.wet_v), _d(p.khtr_u), _d(p.khtr_v), _d(p.dy_cu),
        _d(p.dx_cv), _d(p.idxCu), _d(p.idyCv), _d(p.areaT),
        _d(c["uPoL"]), _d(c["uPoR"]), _i(c["uKoL"]), _i(c["uKoR"]), _d(c["uhEff"]),
        _d(c["vPoL"]), _d(c["vPoR"]), _i(c["vKoL"]), _i(c["vKoR"]), _d(c["vhEff"]), a, b)
    keys = ("add", "mul", "div", "cmp", "cvt")
    return dict(zip(keys, list(a))), dict(zip(keys, list(b)))


def max_threads() -> int:
    return int(lib().redi_oracle_max_threads())
