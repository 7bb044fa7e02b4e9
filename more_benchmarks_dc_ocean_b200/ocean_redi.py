"""Host-side mirror of the reference's ``ocean_redi`` Fortran module over the C-ABI.

Same names, argument order and meaning as redi/ocean_redi.F90:
``OceanRedi`` is ``ocean_redi_t`` (``init``/``destroy``/``enter_data``/
``exit_data``, ``enable``, ``khtr``), and the module functions
``redi_calc_coeffs(grid, metrics, eos, this, ms)`` and
``redi_apply_flux(grid, metrics, this, ms, dt, khtr_u_ext, khtr_v_ext, bc)``
have the reference's gates (silent no-ops where the Fortran returns early).
``HGrid``, ``OceanMetrics``, ``OceanEos``, ``MultilayerState``, ``OceanBC``
mirror the derived types of redi/grid.F90, ocean_metrics.F90, ocean_eos.F90,
multilayer_cgrid_state.F90 and ocean_boundary_types.F90.

Device arrays are torch CUDA float64 tensors laid out as the Fortran arrays
(numpy/torch shape = Fortran shape reversed). torch is only the allocator and
stream provider: every computation runs in the sm_100a kernels of
``libredi_b200.so``; if the library is missing this module raises, it never
falls back to another implementation.
"""

from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libredi_b200.so")

OK, SKIPPED = 0, 1
E_ARG, E_STATE, E_CUDA, E_NOMEM, E_UNSUPPORTED = -1, -2, -3, -4, -5
FP64, MIXED = 0, 1
OBC_WALL = 1

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class RediError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class _Grid(C.Structure):
    _fields_ = [("nx_total", C.c_int), ("ny_total", C.c_int), ("nx_phys", C.c_int), ("ny_phys", C.c_int),
                ("nghost", C.c_int), ("dx", C.c_double), ("dy", C.c_double)]


class _Metrics(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("dy_cu", "dx_cv", "idxCu", "idyCv", "areaT", "wet_u", "wet_v")]


class _Eos(C.Structure):
    _fields_ = [("variant", C.c_int), ("rho0", C.c_double), ("T_ref", C.c_double), ("S_ref", C.c_double),
                ("alpha_T", C.c_double), ("beta_S", C.c_double)]


class _State(C.Structure):
    _fields_ = [("nz_ml", C.c_int), ("idx_temperature", C.c_int), ("idx_salinity", C.c_int),
                ("ntracers", C.c_int), ("h_layer", C.c_void_p), ("hTr", C.POINTER(C.c_void_p))]


class _BC(C.Structure):
    _fields_ = [("west", C.c_int), ("east", C.c_int), ("south", C.c_int), ("north", C.c_int)]


class _Coeffs(C.Structure):
    _fields_ = [("uPoL", C.c_void_p), ("uPoR", C.c_void_p), ("uhEff", C.c_void_p), ("uKoL", C.c_void_p),
                ("uKoR", C.c_void_p), ("vPoL", C.c_void_p), ("vPoR", C.c_void_p), ("vhEff", C.c_void_p),
                ("vKoL", C.c_void_p), ("vKoR", C.c_void_p), ("khtr_u", C.c_void_p), ("khtr_v", C.c_void_p),
                ("nsurf", C.c_int)]


_lib = None


def lib() -> C.CDLL:
    """The sm_100a library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m more_benchmarks_dc_ocean_b200.build` "
                               "(there is no non-CUDA implementation of this path)")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.redi_b200_init.argtypes = [C.POINTER(_Grid), C.c_int, C.c_int, C.POINTER(vp)]
        L.redi_b200_destroy.argtypes = [vp]
        L.redi_b200_set_enable.argtypes = [vp, C.c_int]
        L.redi_b200_set_khtr.argtypes = [vp, C.c_double]
        L.redi_b200_calc_coeffs.argtypes = [C.POINTER(_Grid), C.POINTER(_Metrics), C.POINTER(_Eos), vp,
                                            C.POINTER(_State), vp]
        L.redi_b200_apply_flux.argtypes = [C.POINTER(_Grid), C.POINTER(_Metrics), vp, C.POINTER(_State), C.c_double,
                                           vp, vp, C.POINTER(_BC), vp]
        L.redi_b200_step.argtypes = [C.POINTER(_Grid), C.POINTER(_Metrics), C.POINTER(_Eos), vp, C.POINTER(_State),
                                     C.c_double, vp, vp, C.POINTER(_BC), vp]
        L.redi_b200_get_coeffs.argtypes = [vp, C.POINTER(_Coeffs)]
        L.redi_b200_workspace_bytes.argtypes = [vp]
        L.redi_b200_error_count.argtypes = [vp, C.c_int]
        L.redi_b200_workspace_bytes.restype = C.c_longlong
        L.redi_b200_last_error.restype = C.c_char_p
        L.redi_b200_version.restype = C.c_int
        for name in ("redi_opt_launch", "redi_cuda_launch_"):
            getattr(L, name).restype = None
        _lib = L
    return _lib


def last_error() -> str:
    return lib().redi_b200_last_error().decode()


def _check(rc: int) -> int:
    if rc < 0:
        raise RediError(rc, last_error())
    return rc


def _ptr(t) -> int:
    if t is None:
        return 0
    import torch

    assert isinstance(t, torch.Tensor) and t.is_cuda and t.dtype in (torch.float64, torch.int32), (t.dtype, t.device)
    assert t.is_contiguous()
    return t.data_ptr()


def _stream(stream) -> int:
    import torch

    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


# ---------------------------------------------------------------------------
# Derived types
# ---------------------------------------------------------------------------
@dataclass
class HGrid:
    """hgrid_t (redi/grid.F90:17-25)."""

    nx_total: int
    ny_total: int
    nx_phys: int
    ny_phys: int
    nghost: int = 2
    dx: float = 0.0
    dy: float = 0.0

    def _c(self) -> _Grid:
        return _Grid(self.nx_total, self.ny_total, self.nx_phys, self.ny_phys, self.nghost, self.dx, self.dy)


@dataclass
class OceanMetrics:
    """ocean_metrics_t (redi/ocean_metrics.F90:14-22) on the device."""

    dy_cu: object
    dx_cv: object
    idxCu: object
    idyCv: object
    areaT: object
    wet_u: object
    wet_v: object

    def _c(self) -> _Metrics:
        return _Metrics(*(_ptr(getattr(self, n)) for n in ("dy_cu", "dx_cv", "idxCu", "idyCv", "areaT", "wet_u",
                                                            "wet_v")))


EOS_LINEAR, EOS_WRIGHT_97, EOS_ROQUET_SPV = 1, 2, 4  # redi/ocean_eos.F90:39-51


@dataclass
class OceanEos:
    """ocean_eos_t (redi/ocean_eos.F90:239-278): variant (EOS_LINEAR, EOS_WRIGHT_97,
    EOS_ROQUET_SPV; 0 is taken as LINEAR) and the linear branch's coefficients."""

    rho0: float = 1035.0
    T_ref: float = 10.0
    S_ref: float = 35.0
    alpha_T: float = 1.7e-4
    beta_S: float = 7.6e-4
    variant: int = EOS_LINEAR

    def _c(self) -> _Eos:
        return _Eos(self.variant, self.rho0, self.T_ref, self.S_ref, self.alpha_T, self.beta_S)


@dataclass
class MultilayerState:
    """multilayer_cgrid_state_t (redi/multilayer_cgrid_state.F90:18-28).

    ``idx_temperature``/``idx_salinity`` are 1-based (0 = not registered), as in
    the Fortran; ``tracers`` holds the thickness-weighted hTr tensors.
    """

    nz_ml: int
    h_layer: object
    tracers: List[object] = field(default_factory=list)
    idx_temperature: int = 0
    idx_salinity: int = 0

    def _c(self):
        arr = (C.c_void_p * max(1, len(self.tracers)))(*[_ptr(t) for t in self.tracers])
        st = _State(self.nz_ml, self.idx_temperature, self.idx_salinity, len(self.tracers),
                    _ptr(self.h_layer) if self.h_layer is not None else 0,
                    C.cast(arr, C.POINTER(C.c_void_p)) if self.tracers else None)
        return st, arr


@dataclass
class OceanBC:
    """ocean_bc_state_t (redi/ocean_boundary_types.F90:20-24): bc_type per edge."""

    west: int = OBC_WALL
    east: int = OBC_WALL
    south: int = OBC_WALL
    north: int = OBC_WALL

    def _c(self) -> _BC:
        return _BC(self.west, self.east, self.south, self.north)


class _CudaArray:
    """__cuda_array_interface__ view of a device pointer (aliases, never copies)."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


class OceanRedi:
    """ocean_redi_t (redi/ocean_redi.F90:71-128): Phase-A slots + switches."""

    def __init__(self):
        self._h = C.c_void_p(0)
        self.is_init = False
        self._enable = False
        self._khtr = 0.0
        self.continuous = True
        self.ref_pres = -1.0
        self.nx_total = self.ny_total = self.nz_ml = self.nsurf = 0
        self.precision = FP64

    # -- type-bound procedures --------------------------------------------
    def init(self, grid: HGrid, nz_ml: Optional[int] = None, precision: int = FP64) -> None:
        """ocean_redi_init (ocean_redi.F90:466-507)."""
        if self.is_init:
            self.destroy()
        nz = 1 if nz_ml is None else int(nz_ml)
        h = C.c_void_p(0)
        _check(lib().redi_b200_init(C.byref(grid._c()), nz, int(precision), C.byref(h)))
        self._h = h
        self.is_init = True
        self.nx_total, self.ny_total = grid.nx_total, grid.ny_total
        self.nz_ml = max(1, nz)
        self.nsurf = 2 * self.nz_ml + 2
        self.precision = precision
        self._enable, self._khtr = False, 0.0

    def destroy(self) -> None:
        """ocean_redi_destroy (ocean_redi.F90:509-529)."""
        if self._h:
            lib().redi_b200_destroy(self._h)
        self._h = C.c_void_p(0)
        self.is_init = False
        self.nx_total = self.ny_total = self.nz_ml = self.nsurf = 0

    def enter_data(self) -> None:
        """ocean_redi_enter_data: the slots already live on the device."""

    def exit_data(self) -> None:
        """ocean_redi_exit_data: nothing to unmap."""

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    # -- switches ---------------------------------------------------------
    @property
    def enable(self) -> bool:
        return self._enable

    @enable.setter
    def enable(self, v: bool) -> None:
        self._enable = bool(v)
        if self._h:
            _check(lib().redi_b200_set_enable(self._h, int(bool(v))))

    @property
    def khtr(self) -> float:
        return self._khtr

    @khtr.setter
    def khtr(self, v: float) -> None:
        self._khtr = float(v)
        if self._h:
            _check(lib().redi_b200_set_khtr(self._h, float(v)))

    # -- coefficient slots (device views) -----------------------------------
    def coeffs(self) -> dict:
        """uPoL ... vhEff, khtr_u, khtr_v as torch views of the handle's device slots (FP64 handles).

        The views are writable, so this clears the handle's record of dry faces (faces whose slots
        hold the inert coefficients): the next redi_calc_coeffs rewrites every face. It waits for
        the device."""
        import torch

        c = _Coeffs()
        _check(lib().redi_b200_get_coeffs(self._h, C.byref(c)))
        nx, ny, ns = self.nx_total, self.ny_total, self.nsurf
        out = {}
        for side, (a, b) in (("u", (ny, nx + 1)), ("v", (ny + 1, nx))):
            for n, k, typ in (("PoL", ns, "<f8"), ("PoR", ns, "<f8"), ("KoL", ns, "<i4"), ("KoR", ns, "<i4"),
                              ("hEff", ns - 1, "<f8")):
                out[side + n] = torch.as_tensor(_CudaArray(getattr(c, side + n), (k, a, b), typ), device="cuda")
        out["khtr_u"] = torch.as_tensor(_CudaArray(c.khtr_u, (ny, nx + 1), "<f8"), device="cuda")
        out["khtr_v"] = torch.as_tensor(_CudaArray(c.khtr_v, (ny + 1, nx), "<f8"), device="cuda")
        return out

    def error_count(self, reset: bool = False) -> int:
        """Out-of-order coefficient sublayers seen by Phase B (0 for sweep-produced coefficients)."""
        return _check(lib().redi_b200_error_count(self._h, int(reset))) if self._h else 0

    def workspace_bytes(self) -> int:
        return int(lib().redi_b200_workspace_bytes(self._h)) if self._h else 0


def redi_calc_coeffs(grid: HGrid, metrics: OceanMetrics, eos: OceanEos, this: OceanRedi, ms: MultilayerState,
                     stream=None) -> int:
    """redi_calc_coeffs (ocean_redi.F90:572-607); returns OK or SKIPPED."""
    if not this.is_init:
        return SKIPPED
    st, keep = ms._c()
    return _check(lib().redi_b200_calc_coeffs(C.byref(grid._c()), C.byref(metrics._c()), C.byref(eos._c()),
                                              this._h, C.byref(st), _stream(stream)))


def redi_apply_flux(grid: HGrid, metrics: OceanMetrics, this: OceanRedi, ms: MultilayerState, dt: float,
                    khtr_u_ext=None, khtr_v_ext=None, bc: Optional[OceanBC] = None, stream=None) -> int:
    """redi_apply_flux (ocean_redi.F90:927-1002); returns OK or SKIPPED."""
    if not this.is_init:
        return SKIPPED
    st, keep = ms._c()
    bcs = C.byref(bc._c()) if bc is not None else None
    return _check(lib().redi_b200_apply_flux(C.byref(grid._c()), C.byref(metrics._c()), this._h, C.byref(st),
                                             float(dt), _ptr(khtr_u_ext), _ptr(khtr_v_ext), bcs, _stream(stream)))


def redi_step(grid: HGrid, metrics: OceanMetrics, eos: OceanEos, this: OceanRedi, ms: MultilayerState, dt: float,
              khtr_u_ext=None, khtr_v_ext=None, bc: Optional[OceanBC] = None, stream=None) -> int:
    """redi_calc_coeffs then redi_apply_flux in one call (redi_b200_step): the same results bit for bit,
    with Phase A's column state and the reconstruction of T and S in one pass; returns OK or SKIPPED."""
    if not this.is_init:
        return SKIPPED
    st, keep = ms._c()
    bcs = C.byref(bc._c()) if bc is not None else None
    return _check(lib().redi_b200_step(C.byref(grid._c()), C.byref(metrics._c()), C.byref(eos._c()), this._h,
                                       C.byref(st), float(dt), _ptr(khtr_u_ext), _ptr(khtr_v_ext), bcs,
                                       _stream(stream)))


def redi_opt_launch(nx, ny, nz, dt, nghost, nxp, nyp, walls, eos: OceanEos, h_layer, t_htr, s_htr, wet_u, wet_v,
                    coeffs: dict, khtr_u_ext, khtr_v_ext, khtr_u, khtr_v, dy_cu, dx_cv, idxCu, idyCv, areaT,
                    tr_snap=None, symbol: str = "redi_opt_launch") -> None:
    """Call the reference-compatible launcher export (by-reference scalars, device arrays)."""
    ci = lambda v: C.byref(C.c_int(int(v)))  # noqa: E731
    cd = lambda v: C.byref(C.c_double(float(v)))  # noqa: E731
    ns = 2 * nz + 2
    c = coeffs
    args = [ci(nx), ci(ny), ci(nz), ci(ns), cd(dt), ci(nghost), ci(nxp), ci(nyp)] + [ci(w) for w in walls] + [
        cd(eos.rho0), cd(eos.T_ref), cd(eos.S_ref), cd(eos.alpha_T), cd(eos.beta_S),
        _ptr(h_layer), _ptr(t_htr), _ptr(s_htr), _ptr(wet_u), _ptr(wet_v),
        _ptr(c["uPoL"]), _ptr(c["uPoR"]), _ptr(c["uKoL"]), _ptr(c["uKoR"]), _ptr(c["uhEff"]),
        _ptr(c["vPoL"]), _ptr(c["vPoR"]), _ptr(c["vKoL"]), _ptr(c["vKoR"]), _ptr(c["vhEff"]),
        _ptr(khtr_u_ext), _ptr(khtr_v_ext), _ptr(khtr_u), _ptr(khtr_v),
        _ptr(dy_cu), _ptr(dx_cv), _ptr(idxCu), _ptr(idyCv), _ptr(areaT), _ptr(tr_snap)]
    f = getattr(lib(), symbol)
    f(*[a if not isinstance(a, int) else C.c_void_p(a) for a in args])
    err = last_error()
    if err.startswith(symbol):
        raise RediError(E_ARG, err)


# ---------------------------------------------------------------------------
# Problem <-> device helpers
# ---------------------------------------------------------------------------
@dataclass
class DeviceProblem:
    """A generated RediProblem resident on one GPU, in the mirrored types."""

    grid: HGrid
    metrics: OceanMetrics
    eos: OceanEos
    ms: MultilayerState
    khtr_u_ext: object
    khtr_v_ext: object
    bc: OceanBC
    dt: float


def to_device(p, device="cuda", tracers: Optional[Sequence[np.ndarray]] = None) -> DeviceProblem:
    """Upload a ``more_benchmarks_dc_ocean_b200.inputs.RediProblem``."""
    import torch

    def d(a):
        return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(device)

    trs = [d(t) for t in (tracers if tracers is not None else p.tracers)]
    ww, we, ws, wn = p.walls
    wall = lambda f: OBC_WALL if f else 0  # noqa: E731
    return DeviceProblem(
        grid=HGrid(p.nx, p.ny, p.nx_phys, p.ny_phys, p.nghost, 0.0, 0.0),
        metrics=OceanMetrics(d(p.dy_cu), d(p.dx_cv), d(p.idxCu), d(p.idyCv), d(p.areaT), d(p.wet_u), d(p.wet_v)),
        eos=OceanEos(p.eos.rho0, p.eos.T_ref, p.eos.S_ref, p.eos.alpha_T, p.eos.beta_S,
                     getattr(p.eos, "variant", EOS_LINEAR)),
        ms=MultilayerState(p.nz, d(p.h), trs, p.idx_temperature + 1, p.idx_salinity + 1),
        khtr_u_ext=d(p.khtr_u), khtr_v_ext=d(p.khtr_v),
        bc=OceanBC(wall(ww), wall(we), wall(ws), wall(wn)), dt=p.dt)


def _hptr(t) -> int:
    import torch

    assert isinstance(t, torch.Tensor) and not t.is_cuda and t.dtype == torch.float64 and t.is_contiguous(), t
    return t.data_ptr()


def redi_step_host(grid: HGrid, metrics: OceanMetrics, eos: OceanEos, this: OceanRedi, ms_host: MultilayerState,
                   dt: float, khtr_u_ext=None, khtr_v_ext=None, bc: Optional[OceanBC] = None, nbands: int = 8,
                   stream=None) -> int:
    """redi_calc_coeffs + redi_apply_flux on a host-resident state (h and tracers are CPU float64
    tensors, page-locked for overlap), pipelined over ``nbands`` row bands; stream-ordered."""
    if not this.is_init:
        return SKIPPED
    L = lib()
    L.redi_b200_step_host.argtypes = [C.POINTER(_Grid), C.POINTER(_Metrics), C.POINTER(_Eos), C.c_void_p,
                                      C.POINTER(_State), C.c_double, C.c_void_p, C.c_void_p, C.POINTER(_BC),
                                      C.c_int, C.c_void_p]
    arr = (C.c_void_p * max(1, len(ms_host.tracers)))(*[_hptr(t) for t in ms_host.tracers])
    st = _State(ms_host.nz_ml, ms_host.idx_temperature, ms_host.idx_salinity, len(ms_host.tracers),
                _hptr(ms_host.h_layer), C.cast(arr, C.POINTER(C.c_void_p)) if ms_host.tracers else None)
    return _check(L.redi_b200_step_host(C.byref(grid._c()), C.byref(metrics._c()), C.byref(eos._c()), this._h,
                                        C.byref(st), float(dt), _ptr(khtr_u_ext), _ptr(khtr_v_ext),
                                        C.byref(bc._c()) if bc is not None else None, int(nbands), _stream(stream)))


def eos_points(eos: OceanEos, T, S, p, stream=None):
    """eos_density_point + eos_specvol_derivs (redi/ocean_eos.F90:450-546) at every point of the
    float64 CUDA tensors T, S, p (Pa); returns (rho, dsv_dt, dsv_ds) tensors."""
    import torch

    L = lib()
    L.redi_b200_eos_points.argtypes = [C.POINTER(_Eos), C.c_int] + [C.c_void_p] * 7
    T, S, p = (t.contiguous() for t in (T, S, p))
    out = [torch.empty_like(T) for _ in range(3)]
    e = eos._c()
    _check(L.redi_b200_eos_points(C.byref(e), T.numel(), _ptr(T), _ptr(S), _ptr(p), *[_ptr(o) for o in out],
                                  _stream(stream)))
    return tuple(out)


def make_redi(dp: DeviceProblem, precision: int = FP64) -> OceanRedi:
    r = OceanRedi()
    r.init(dp.grid, dp.ms.nz_ml, precision)
    r.enable = True
    return r


def step(dp: DeviceProblem, redi: OceanRedi, nsteps: int = 1, stream=None) -> None:
    """``nsteps`` Redi steps (Phase A, then Phase B on every tracer: redi_step), stream-ordered."""
    for _ in range(nsteps):
        redi_step(dp.grid, dp.metrics, dp.eos, redi, dp.ms, dp.dt, dp.khtr_u_ext, dp.khtr_v_ext, dp.bc, stream)


# ---------------------------------------------------------------------------
# Many domains in one persistent launch (no counterpart in the reference)
# ---------------------------------------------------------------------------
STATUS_TIMEOUT = 1
STAGE_NAMES = ("column_state", "neutral_sweep", "tracer_recon")


class _Domain(C.Structure):
    _fields_ = [("grid", _Grid), ("metrics", _Metrics), ("eos", _Eos), ("ms", _State),
                ("khtr_u_ext", C.c_void_p), ("khtr_v_ext", C.c_void_p), ("bc", _BC), ("dt", C.c_double)]


def _batch_lib() -> C.CDLL:
    L = lib()
    if not getattr(L, "_batch_types", False):
        vp = C.c_void_p
        L.redi_b200_batch_create.argtypes = [C.c_int, C.POINTER(_Domain), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                             C.POINTER(vp)]
        L.redi_b200_batch_step.argtypes = [vp, vp]
        L.redi_b200_batch_status.argtypes = [vp, _ip, _ip, _ip, _ip]
        L.redi_b200_batch_set_wait_limit.argtypes = [vp, C.c_longlong]
        L.redi_b200_batch_hold.argtypes = [vp, C.c_int, C.c_int]
        L.redi_b200_batch_set_tuning.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int]
        L.redi_b200_batch_get_tuning.argtypes = [vp, _ip, _ip, _ip, _ip, _ip]
        L.redi_b200_batch_set_accounting.argtypes = [vp, C.c_int]
        L.redi_b200_batch_stage_times.argtypes = [vp, _dp, _dp, C.POINTER(C.c_longlong)]
        L.redi_b200_batch_updates.argtypes = [vp]
        L.redi_b200_batch_updates.restype = C.c_longlong
        L.redi_b200_batch_items.argtypes = [vp]
        L.redi_b200_batch_items.restype = C.c_longlong
        L.redi_b200_batch_destroy.argtypes = [vp]
        L._batch_types = True
    return L


def stage_name(stage: int) -> str:
    """Name of a stage index reported by ``RediBatch.status``."""
    if stage < 3:
        return STAGE_NAMES[stage]
    g, kind = divmod(stage - 3, 2)
    return f"{'face_flux' if kind == 0 else 'cell_gather'}[pair {g}]"


class RediBatch:
    """Independent regional domains stepped together by one persistent kernel.

    ``domains`` are ``DeviceProblem``s (per-face diffusivities required); their
    tensors must stay alive while the batch exists, their device addresses are
    baked into it. Each ``step`` runs ``redi_calc_coeffs`` + ``redi_apply_flux``
    on every domain; per domain the result equals the handle API's at the same
    precision, bit for bit.
    """

    def __init__(self, domains: Sequence[DeviceProblem], precision: int = FP64, tile=(32, 4), chunk: int = 8,
                 use_graph: bool = True):
        L = _batch_lib()
        self.domains = list(domains)
        self.precision = precision
        self.tile = tuple(tile)
        self.chunk = chunk
        self.use_graph = bool(use_graph)
        arr = (_Domain * len(self.domains))()
        keep = []
        for k, dp in enumerate(self.domains):
            st, tr = dp.ms._c()
            keep.append(tr)
            arr[k] = _Domain(dp.grid._c(), dp.metrics._c(), dp.eos._c(), st, _ptr(dp.khtr_u_ext), _ptr(dp.khtr_v_ext),
                             dp.bc._c(), float(dp.dt))
        h = C.c_void_p()
        _check(L.redi_b200_batch_create(len(self.domains), arr, precision, int(tile[0]), int(tile[1]), int(chunk),
                                        int(self.use_graph), C.byref(h)))
        self._h = h

    def step(self, nsteps: int = 1, stream=None) -> None:
        s = _stream(stream)
        for _ in range(nsteps):
            _check(_batch_lib().redi_b200_batch_step(self._h, s))

    def status(self) -> dict:
        """Outcome of the last step (synchronises)."""
        st, d, sg, bad = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        _check(_batch_lib().redi_b200_batch_status(self._h, C.byref(st), C.byref(d), C.byref(sg), C.byref(bad)))
        out = {"status": st.value, "bad": bad.value}
        if st.value:
            out.update(domain=d.value, stage=sg.value, stage_name=stage_name(sg.value))
        return out

    def set_wait_limit(self, ns: int) -> None:
        _check(_batch_lib().redi_b200_batch_set_wait_limit(self._h, int(ns)))

    def set_tuning(self, tile, chunk: int, occupancy: int = 0) -> None:
        """Gather tile (bx, by), bx * by = 128, vertical chunk (4, 8, 16) and register budget
        (blocks per SM: 4, 5, 6; 0 keeps it); results do not depend on it."""
        _check(_batch_lib().redi_b200_batch_set_tuning(self._h, int(tile[0]), int(tile[1]), int(chunk),
                                                       int(occupancy)))
        self.tile, self.chunk = tuple(tile), chunk

    def get_tuning(self) -> dict:
        bx, by, ch, occ, grid = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_int()
        _check(_batch_lib().redi_b200_batch_get_tuning(self._h, C.byref(bx), C.byref(by), C.byref(ch), C.byref(occ),
                                                       C.byref(grid)))
        return {"tile": (bx.value, by.value), "chunk": ch.value, "occupancy": occ.value, "grid": grid.value}

    def set_accounting(self, on: bool = True) -> None:
        _check(_batch_lib().redi_b200_batch_set_accounting(self._h, int(bool(on))))

    def stage_times(self) -> dict:
        """Per stage kind of the last step (accounting on): wait / busy ms summed over blocks, tiles."""
        w, b, t = (C.c_double * 5)(), (C.c_double * 5)(), (C.c_longlong * 5)()
        _check(_batch_lib().redi_b200_batch_stage_times(self._h, w, b, t))
        names = ("column_state", "neutral_sweep", "tracer_recon", "face_flux", "cell_gather")
        return {n: {"wait_ms": w[k], "busy_ms": b[k], "tiles": t[k]} for k, n in enumerate(names)}

    def hold(self, domain: int, hold: bool = True) -> None:
        _check(_batch_lib().redi_b200_batch_hold(self._h, int(domain), int(bool(hold))))

    @property
    def updates(self) -> int:
        return int(_batch_lib().redi_b200_batch_updates(self._h))

    @property
    def items(self) -> int:
        return int(_batch_lib().redi_b200_batch_items(self._h))

    def destroy(self) -> None:
        if getattr(self, "_h", None):
            _batch_lib().redi_b200_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:  # pragma: no cover - interpreter shutdown
            pass
