"""Host-side mirror of the reference's ALE remap module over the C-ABI (include/ale_b200.h).

Same names, argument order and meaning as ale_remap/ale_remap.F90 and
ale_remap/remap_state.F90: ``ale_remap_step(grid, vcoord, ms, bt_eta, bt_H_ref)``
with ``AleGrid`` (``hgrid_t``), ``OceanVcoord`` (``ocean_vcoord_t``: coord_type,
remap_method, remap_vel_conserve_ke, dsig and the remap workspaces) and
``AleState`` (``multilayer_cgrid_state_t``: h_layer, the tracer slots, the face
velocities and the three budgets). ``ale_remap_step_opt`` is the same function
(the reference's optimized form is bit-identical to it).

``ale_remap_cuda`` and ``ale_remap_opt`` call the exports with the reference
launchers' signatures.

Arrays are torch CUDA float64 tensors in the Fortran shapes reversed (layers
(nz, ny, nx), u faces (nz, ny, nx+1), v faces (nz, ny+1, nx), cells (ny, nx)).
Every computation runs in the sm_100a kernels of ``libredi_b200.so``.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional

from .ocean_redi import lib as _redi_lib

OK = 0
E_ARG, E_CUDA, E_UNSUPPORTED = -1, -3, -5
REMAP_PCM, REMAP_PLM, REMAP_PPM, REMAP_PPM_H4, REMAP_PQM = 1, 2, 3, 4, 5
VCOORD_SIGMA, VCOORD_ZSTAR = 2, 3  # ale_remap/constants.F90:28-33


class AleError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class StepArgs(C.Structure):
    """``ale_b200_step_args`` (include/ale_b200.h)."""

    _fields_ = ([(n, C.c_int) for n in ("nx", "ny", "nz", "method", "conserve_ke", "ntracers", "idx_temperature",
                                        "idx_salinity")] +
                [("h_layer", C.c_void_p), ("tracers", C.POINTER(C.c_void_p))] +
                [(n, C.c_void_p) for n in ("u", "v", "mass_budget", "heat_budget", "salt_budget", "bt_eta",
                                           "bt_H_ref", "dsig", "total_h", "h_ref", "h_old", "target_h")])


_bound = False


def lib() -> C.CDLL:
    global _bound
    L = _redi_lib()
    if not _bound:
        L.ale_b200_remap_step.argtypes = [C.POINTER(StepArgs), C.c_void_p]
        L.ale_b200_last_error.restype = C.c_char_p
        p = C.c_void_p
        L.ale_remap_cuda.argtypes = [C.c_int] * 5 + [p] * 15
        L.ale_remap_cuda.restype = None
        L.ale_remap_opt.argtypes = [C.c_int] * 3 + [p] * 13
        L.ale_remap_opt.restype = None
        L.cuda_sync.restype = None
        _bound = True
    return L


def last_error() -> str:
    return lib().ale_b200_last_error().decode()


def _ptr(t):
    return None if t is None else t.data_ptr()


@dataclass
class AleGrid:
    """``hgrid_t`` (ale_remap/remap_state.F90:17-20)."""

    nx_total: int
    ny_total: int


@dataclass
class OceanVcoord:
    """``ocean_vcoord_t`` (ale_remap/remap_state.F90:28-41)."""

    nz_ml: int
    dsig: object
    target_h: object
    remap_h_old: object
    remap_total_h: object
    remap_h_ref: object
    coord_type: int = VCOORD_ZSTAR
    is_init: bool = True
    nx_total: int = 0
    ny_total: int = 0
    remap_method: int = REMAP_PPM
    regrid_time_scale: float = 0.0
    remap_vel_conserve_ke: bool = False


@dataclass
class AleState:
    """``multilayer_cgrid_state_t`` for the remap (ale_remap/remap_state.F90:43-55); tracer slots may be None."""

    nz_ml: int
    h_layer: object
    tracers: List[Optional[object]]
    u_face_x_layer: Optional[object]
    v_face_y_layer: Optional[object]
    mass_budget_remap: object
    heat_budget_remap: object
    salt_budget_remap: object
    idx_temperature: int = 1  # 1-based, as the Fortran
    idx_salinity: int = 2
    _keep: list = field(default_factory=list, repr=False)


def _args(nx, ny, nz, method, conserve_ke, h_layer, tracers, idx_t, idx_s, u, v, mass_b, heat_b, salt_b, bt_eta,
          bt_H_ref, dsig, total_h, h_ref, h_old, target_h):
    a = StepArgs()
    a.nx, a.ny, a.nz, a.method, a.conserve_ke = nx, ny, nz, int(method), int(bool(conserve_ke))
    a.ntracers, a.idx_temperature, a.idx_salinity = len(tracers), idx_t, idx_s
    tab = (C.c_void_p * max(1, len(tracers)))(*[_ptr(t) for t in tracers])
    a.tracers = C.cast(tab, C.POINTER(C.c_void_p))
    a.h_layer = _ptr(h_layer)
    for n, t in (("u", u), ("v", v), ("mass_budget", mass_b), ("heat_budget", heat_b), ("salt_budget", salt_b),
                 ("bt_eta", bt_eta), ("bt_H_ref", bt_H_ref), ("dsig", dsig), ("total_h", total_h), ("h_ref", h_ref),
                 ("h_old", h_old), ("target_h", target_h)):
        setattr(a, n, _ptr(t))
    return a, tab


def ale_remap_step(grid: AleGrid, vcoord: OceanVcoord, ms: AleState, bt_eta, bt_H_ref, stream=None) -> None:
    """One ALE remap step (ale_remap/ale_remap.F90:76-188), stream-ordered on ``stream`` (default: torch's).

    Like the reference's transcription it supports the zstar / sigma target
    (the only coordinates its configurations use) and ignores
    regrid_time_scale (its time filter is off by default and dropped there)."""
    import torch

    if vcoord.coord_type not in (VCOORD_SIGMA, VCOORD_ZSTAR):
        raise AleError(E_UNSUPPORTED, "ale_remap_step: only the zstar / sigma target is implemented")
    if not vcoord.is_init:
        raise AleError(E_ARG, "ale_remap_step: vcoord is not initialised")
    faces = ms.u_face_x_layer is not None and ms.v_face_y_layer is not None
    a, tab = _args(grid.nx_total, grid.ny_total, ms.nz_ml, vcoord.remap_method, vcoord.remap_vel_conserve_ke,
                   ms.h_layer, ms.tracers, ms.idx_temperature - 1, ms.idx_salinity - 1,
                   ms.u_face_x_layer if faces else None, ms.v_face_y_layer if faces else None,
                   ms.mass_budget_remap, ms.heat_budget_remap, ms.salt_budget_remap, bt_eta, bt_H_ref, vcoord.dsig,
                   vcoord.remap_total_h, vcoord.remap_h_ref, vcoord.remap_h_old, vcoord.target_h)
    st = stream if stream is not None else torch.cuda.current_stream()
    rc = lib().ale_b200_remap_step(C.byref(a), C.c_void_p(st.cuda_stream))
    if rc < 0:
        raise AleError(rc, last_error())


ale_remap_step_opt = ale_remap_step


def ale_remap_cuda(nx, ny, nz, method, fused, h_layer, h_old, target_h, total_h, h_ref, hTr_t, hTr_s, u, v, mass_b,
                   heat_b, salt_b, eta, H_ref, dsig) -> None:
    """The export with ale_remap/ale_kernel.cu:453's signature (asynchronous on the legacy stream)."""
    lib().ale_remap_cuda(nx, ny, nz, method, fused, *[_ptr(t) for t in (
        h_layer, h_old, target_h, total_h, h_ref, hTr_t, hTr_s, u, v, mass_b, heat_b, salt_b, eta, H_ref, dsig)])


def ale_remap_opt(nx, ny, nz, h_layer, h_old, target_h, hTr_t, hTr_s, u, v, mass_b, heat_b, salt_b, eta, H_ref,
                  dsig) -> None:
    """The export with ale_remap/opt_kernel.cu:399's signature (asynchronous on the legacy stream)."""
    lib().ale_remap_opt(nx, ny, nz, *[_ptr(t) for t in (
        h_layer, h_old, target_h, hTr_t, hTr_s, u, v, mass_b, heat_b, salt_b, eta, H_ref, dsig)])


# ---- AleProblem helpers (more_benchmarks_dc_ocean_b200.ale_inputs) ----------
def to_device(p, device="cuda"):
    """The arrays of an ``AleProblem`` as device tensors: a dict, tracers under 'tracers'."""
    import torch

    d = lambda a: None if a is None else torch.from_numpy(a).to(device)  # noqa: E731
    out = {k: d(getattr(p, k)) for k in ("h_layer", "u", "v", "mass_budget", "heat_budget", "salt_budget", "bt_eta",
                                        "bt_H_ref", "dsig", "total_h", "h_ref", "h_old", "target_h")}
    out["tracers"] = [d(t) for t in p.tracers]
    return out


def step_problem(p, d, nsteps: int = 1, stream=None) -> None:
    """nsteps steps of an ``AleProblem`` on its device arrays ``d``."""
    import torch

    a, tab = _args(p.nx, p.ny, p.nz, p.method, p.conserve_ke, d["h_layer"], d["tracers"], p.idx_temperature,
                   p.idx_salinity, d["u"], d["v"], d["mass_budget"], d["heat_budget"], d["salt_budget"], d["bt_eta"],
                   d["bt_H_ref"], d["dsig"], d["total_h"], d["h_ref"], d["h_old"], d["target_h"])
    st = stream if stream is not None else torch.cuda.current_stream()
    for _ in range(nsteps):
        rc = lib().ale_b200_remap_step(C.byref(a), C.c_void_p(st.cuda_stream))
        if rc < 0:
            raise AleError(rc, last_error())


def host_arrays(d):
    """Device arrays back to numpy, keyed like ``AleProblem.arrays()``."""
    out = {k: v.cpu().numpy() for k, v in d.items() if k not in ("tracers", "bt_H_ref", "dsig") and v is not None}
    for n, t in enumerate(d["tracers"]):
        if t is not None:
            out[f"tracer{n}"] = t.cpu().numpy()
    return out
