"""TEST INFRASTRUCTURE ONLY: ctypes front end of the MEKE CPU oracle (meke_oracle.cpp).

``step(problem, nsteps)`` runs meke_step_ext (meke/meke.F90:60-131) in place on
the numpy arrays of a ``MekeProblem``. Only tests, smoke() and the CPU
baseline of bench.py use it, as the checker.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libmeke_oracle.so")

_PTRS = ("meke", "kh_diff", "le", "ku", "i_mass", "depth_tot", "bottom_fac2", "barotr_fac2", "src", "uflux",
         "vflux", "mass_ws", "rd_ws", "sn_u_ws", "sn_v_ws", "ke_diss_ws", "u_bbl2", "f_centre", "gm_src",
         "ke_diss_ext", "h_layer", "rho_layer", "areaT", "iareaT", "idxT", "idyT", "dy_cu", "dx_cv", "idxCu",
         "idyCv")
_DBL = ("dt", "dtscale", "cd_scale", "cb", "ct", "min_gamma2", "cdrag", "uscale", "a_deform", "a_rhines", "a_eady",
        "a_frict", "a_grid", "bgsrc", "gmcoeff", "frcoeff", "damping", "kh_bg", "k4", "khmeke_fac", "khcoeff",
        "visc_coeff_ku", "rho0")


class _Args(C.Structure):
    _fields_ = ([(n, C.c_void_p) for n in _PTRS] + [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int)] +
                [(n, C.c_double) for n in _DBL] + [("backscatter", C.c_int), ("del2", C.c_void_p)])


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            subprocess.run(["make", "-s", "-C", HERE], check=True)
        _lib = C.CDLL(LIB)
        _lib.meke_oracle_step.argtypes = [C.POINTER(_Args)]
        _lib.meke_oracle_step.restype = C.c_int
    return _lib


def step(p, nsteps: int = 1) -> None:
    """nsteps MEKE steps of problem p, in place."""
    L = lib()
    for k, v in p.arrays.items():
        assert v.dtype == np.float64 and v.flags.c_contiguous, k
    a = _Args()
    for n in _PTRS:
        setattr(a, n, p.arrays[n].ctypes.data)
    a.del2 = p.arrays["del2"].ctypes.data
    a.nx, a.ny, a.nz = p.nx, p.ny, p.nz
    for n in _DBL:
        setattr(a, n, float(p.config[n]))
    a.backscatter = int(p.config["backscatter"])
    for _ in range(nsteps):
        rc = L.meke_oracle_step(C.byref(a))
        if rc != 0:
            raise RuntimeError(f"meke oracle: status {rc}")
