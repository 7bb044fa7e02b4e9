"""TEST INFRASTRUCTURE ONLY: ctypes front end of the ALE remap CPU oracle (ale_oracle.cpp).

``step(problem, nsteps)`` runs ale_remap_step (ale_remap/ale_remap.F90:76-188)
in place on the numpy arrays of an ``AleProblem``. Only tests, smoke() and the
CPU baseline of bench.py use it, as the checker.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libale_oracle.so")


class _Args(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("nx", "ny", "nz", "method", "conserve_ke", "ntracers", "idx_temperature",
                                       "idx_salinity")] + \
               [("h_layer", C.c_void_p), ("tracers", C.POINTER(C.c_void_p)), ("u", C.c_void_p), ("v", C.c_void_p),
                ("mass_budget", C.c_void_p), ("heat_budget", C.c_void_p), ("salt_budget", C.c_void_p),
                ("bt_eta", C.c_void_p), ("bt_H_ref", C.c_void_p), ("dsig", C.c_void_p), ("total_h", C.c_void_p),
                ("h_ref", C.c_void_p), ("h_old", C.c_void_p), ("target_h", C.c_void_p)]


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            subprocess.run(["make", "-s", "-C", HERE], check=True)
        _lib = C.CDLL(LIB)
        _lib.ale_oracle_step.argtypes = [C.POINTER(_Args)]
        _lib.ale_oracle_step.restype = C.c_int
    return _lib


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data


def step(p, nsteps: int = 1) -> None:
    """nsteps ALE remap steps of problem p, in place."""
    L = lib()
    a = _Args()
    a.nx, a.ny, a.nz, a.method, a.conserve_ke = p.nx, p.ny, p.nz, p.method, int(p.conserve_ke)
    a.ntracers = len(p.tracers)
    a.idx_temperature, a.idx_salinity = p.idx_temperature, p.idx_salinity
    tab = (C.c_void_p * max(1, len(p.tracers)))(*[_p(t) for t in p.tracers])
    a.tracers = C.cast(tab, C.POINTER(C.c_void_p))
    for n in ("h_layer", "u", "v", "mass_budget", "heat_budget", "salt_budget", "bt_eta", "bt_H_ref", "dsig",
              "total_h", "h_ref", "h_old", "target_h"):
        setattr(a, n, _p(getattr(p, n)))
    for _ in range(nsteps):
        rc = L.ale_oracle_step(C.byref(a))
        if rc != 0:
            raise RuntimeError(f"ale oracle: status {rc}")
