"""Host-side mirror of the reference's MEKE step over the C-ABI (include/meke_b200.h).

Same names, argument order and meaning as meke/meke.F90 and meke/meke_state.F90:
``OceanMeke`` is ``ocean_meke_t`` (its scalars with the production defaults and
its arrays), ``MekeMetrics`` / ``MekeLayers`` / ``OceanGM`` are the parts of
``ocean_metrics_t`` / ``multilayer_cgrid_state_t`` / ``ocean_gm_t`` the step
reads, and ``meke_step_ext(nx, ny, nz, m, metrics, gm, ms, dt, ke_diss_ext)``
is the step (``meke_step_ext_fused`` is the same function: the reference's
fused form is bit-identical to it).

``meke_cuda_launch`` and ``meke_opt_launch`` call the exports with the
reference launchers' signatures on a ``MekeArgs`` block.

Arrays are torch CUDA float64 tensors in the Fortran shapes reversed (cell
fields (ny, nx), u faces (ny, nx+1), v faces (ny+1, nx), layers (nz, ny, nx)).
Every computation runs in the sm_100a kernels of ``libredi_b200.so``; there is
no other implementation to fall back to.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Dict, Optional

from .ocean_redi import lib as _redi_lib

OK = 0
E_ARG, E_CUDA, E_NOMEM = -1, -3, -4

_PTRS = ("meke", "kh_diff", "le", "ku", "i_mass", "depth_tot", "bottom_fac2", "barotr_fac2", "src", "uflux",
         "vflux", "mass_ws", "rd_ws", "sn_u_ws", "sn_v_ws", "ke_diss_ws", "u_bbl2", "f_centre", "gm_src",
         "ke_diss_ext", "h_layer", "rho_layer", "areaT", "iareaT", "idxT", "idyT", "dy_cu", "dx_cv", "idxCu",
         "idyCv")
_DBL = ("dt", "dtscale", "cd_scale", "cb", "ct", "min_gamma2", "cdrag", "uscale", "a_deform", "a_rhines", "a_eady",
        "a_frict", "a_grid", "bgsrc", "gmcoeff", "frcoeff", "damping", "kh_bg", "k4", "khmeke_fac", "khcoeff",
        "visc_coeff_ku", "rho0")


class MekeArgs(C.Structure):
    """``struct MekeArgs`` (meke/meke_args.h:38-52), field for field."""

    _fields_ = ([(n, C.c_void_p) for n in _PTRS] + [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int)] +
                [(n, C.c_double) for n in _DBL] + [("backscatter", C.c_int)])


class MekeError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


_bound = False


def lib() -> C.CDLL:
    global _bound
    L = _redi_lib()
    if not _bound:
        L.meke_b200_create.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]
        L.meke_b200_destroy.argtypes = [C.c_void_p]
        L.meke_b200_step.argtypes = [C.c_void_p, C.POINTER(MekeArgs), C.c_void_p, C.c_void_p]
        L.meke_b200_scratch_energy.argtypes = [C.c_void_p]
        L.meke_b200_scratch_energy.restype = C.c_void_p
        L.meke_b200_last_error.restype = C.c_char_p
        L.meke_cuda_launch.argtypes = [C.POINTER(MekeArgs), C.c_int]
        L.meke_cuda_launch.restype = None
        L.meke_cuda_graph_reset.restype = None
        L.meke_opt_launch.argtypes = [C.POINTER(MekeArgs), C.c_void_p]
        L.meke_opt_launch.restype = None
        _bound = True
    return L


def _check(rc: int) -> int:
    if rc < 0:
        raise MekeError(rc, lib().meke_b200_last_error().decode())
    return rc


def _ptr(t) -> Optional[int]:
    return None if t is None else t.data_ptr()


@dataclass
class MekeMetrics:
    """The ``ocean_metrics_t`` fields the step reads (meke/meke_state.F90:27-36)."""

    areaT: object
    iareaT: object
    idxT: object
    idyT: object
    dy_cu: object
    dx_cv: object
    idxCu: object
    idyCv: object


@dataclass
class MekeLayers:
    """``multilayer_cgrid_state_t`` for the step (meke/meke_state.F90:38-42)."""

    nz_ml: int
    h_layer: object
    rho_layer: object


@dataclass
class OceanGM:
    """``ocean_gm_t`` (meke/meke_state.F90:44-48)."""

    gm_src: object
    rho0: float = 1035.0
    is_init: bool = True


@dataclass
class OceanMeke:
    """``ocean_meke_t`` (meke/meke_state.F90:52-105): scalars with the production defaults, and arrays."""

    is_init: bool = False
    enable: bool = False
    gmcoeff: float = -1.0
    frcoeff: float = -1.0
    bgsrc: float = 0.0
    damping: float = 0.0
    kh: float = -1.0
    k4: float = -1.0
    khmeke_fac: float = 0.0
    advection_factor: float = 0.0
    khcoeff: float = 1.0
    cd_scale: float = 0.0
    cb: float = 25.0
    ct: float = 50.0
    min_gamma2: float = 1.0e-4
    uscale: float = 0.0
    dtscale: float = 1.0
    cdrag: float = 2.5e-3
    use_bbl_drag: bool = False
    alpha_deform: float = 0.0
    alpha_rhines: float = 0.0
    alpha_eady: float = 0.0
    alpha_frict: float = 0.0
    alpha_grid: float = 0.0
    khth_fac: float = 0.0
    khtr_fac: float = 0.0
    backscatter: bool = False
    visc_coeff_ku: float = 0.0
    nx_total: int = 0
    ny_total: int = 0
    nz_ml: int = 0
    arrays: Dict[str, object] = field(default_factory=dict)
    _handle: Optional[int] = field(default=None, repr=False)

    ARRAYS = ("meke", "kh_diff", "le", "ku", "i_mass", "depth_tot", "bottom_fac2", "barotr_fac2", "src", "uflux",
              "vflux", "del2", "mass_ws", "u_bbl2", "ke_diss_ws", "rd_ws", "f_centre", "sn_u_ws", "sn_v_ws")

    def init(self, nx: int, ny: int, nz: int, device="cuda") -> "OceanMeke":
        """Allocates the arrays (zeros) for an nx x ny domain with nz layers."""
        import torch

        self.nx_total, self.ny_total, self.nz_ml = nx, ny, nz
        z = lambda *s: torch.zeros(s, dtype=torch.float64, device=device)  # noqa: E731
        for n in self.ARRAYS:
            self.arrays[n] = z(ny, nx + 1) if n in ("uflux", "sn_u_ws") else z(ny + 1, nx) if n in (
                "vflux", "sn_v_ws") else z(ny, nx)
        self.is_init = True
        return self

    def __getattr__(self, name):
        arrays = self.__dict__.get("arrays", {})
        if name in arrays:
            return arrays[name]
        raise AttributeError(name)

    def destroy(self) -> None:
        if self._handle:
            lib().meke_b200_destroy(self._handle)
            self._handle = None

    def handle(self) -> int:
        if self._handle is None:
            h = C.c_void_p()
            _check(lib().meke_b200_create(self.nx_total, self.ny_total, self.nz_ml, C.byref(h)))
            self._handle = h.value
        return self._handle


def make_args(nx: int, ny: int, nz: int, arrays: Dict[str, object], config: Dict[str, float]) -> MekeArgs:
    """A ``MekeArgs`` block over device tensors (``arrays`` by MekeArgs name) and scalars."""
    a = MekeArgs()
    for n in _PTRS:
        setattr(a, n, _ptr(arrays.get(n)))
    a.nx, a.ny, a.nz = nx, ny, nz
    for n in _DBL:
        setattr(a, n, float(config[n]))
    a.backscatter = int(config["backscatter"])
    return a


def meke_step_ext(nx: int, ny: int, nz: int, m: OceanMeke, metrics: MekeMetrics, gm: OceanGM, ms: MekeLayers,
                  dt: float, ke_diss_ext, stream=None) -> None:
    """One MEKE step (meke/meke.F90:60-131), stream-ordered on ``stream`` (default: torch's current stream).

    Like the reference's ``meke_step_ext`` it ignores advection_factor,
    use_bbl_drag (u_bbl2 is read as it stands), khth_fac and khtr_fac.
    """
    import torch

    arrays = dict(m.arrays)
    arrays.update(metrics.__dict__)
    arrays.update(h_layer=ms.h_layer, rho_layer=ms.rho_layer, gm_src=gm.gm_src, ke_diss_ext=ke_diss_ext)
    config = dict(dt=dt, dtscale=m.dtscale, cd_scale=m.cd_scale, cb=m.cb, ct=m.ct, min_gamma2=m.min_gamma2,
                  cdrag=m.cdrag, uscale=m.uscale, a_deform=m.alpha_deform, a_rhines=m.alpha_rhines,
                  a_eady=m.alpha_eady, a_frict=m.alpha_frict, a_grid=m.alpha_grid, bgsrc=m.bgsrc,
                  gmcoeff=m.gmcoeff, frcoeff=m.frcoeff, damping=m.damping, kh_bg=m.kh, k4=m.k4,
                  khmeke_fac=m.khmeke_fac, khcoeff=m.khcoeff, visc_coeff_ku=m.visc_coeff_ku, rho0=gm.rho0,
                  backscatter=int(m.backscatter))
    args = make_args(nx, ny, nz, arrays, config)
    st = stream if stream is not None else torch.cuda.current_stream()
    _check(lib().meke_b200_step(m.handle(), C.byref(args), _ptr(m.arrays.get("del2")), C.c_void_p(st.cuda_stream)))


meke_step_ext_fused = meke_step_ext


def meke_cuda_launch(args: MekeArgs, mode: int) -> None:
    """The export with meke/meke_args.h:61's signature (synchronous)."""
    lib().meke_cuda_launch(C.byref(args), int(mode))


def meke_cuda_graph_reset() -> None:
    lib().meke_cuda_graph_reset()


def meke_opt_launch(args: MekeArgs, meke_scratch) -> None:
    """The export with meke/opt_kernel.cu:274's signature (synchronous)."""
    lib().meke_opt_launch(C.byref(args), _ptr(meke_scratch))


def last_error() -> str:
    return lib().meke_b200_last_error().decode()


def to_device(p, device="cuda") -> Dict[str, object]:
    """The arrays of a ``MekeProblem`` as device tensors, by MekeArgs name."""
    import torch

    return {k: torch.from_numpy(v).to(device) for k, v in p.arrays.items()}


def step_problem(p, d: Dict[str, object], nsteps: int = 1, handle: Optional[int] = None, stream=None) -> int:
    """nsteps steps of a ``MekeProblem`` on its device arrays ``d``; returns the handle used."""
    import torch

    L = lib()
    if handle is None:
        h = C.c_void_p()
        _check(L.meke_b200_create(p.nx, p.ny, p.nz, C.byref(h)))
        handle = h.value
    args = make_args(p.nx, p.ny, p.nz, d, p.config)
    st = stream if stream is not None else torch.cuda.current_stream()
    for _ in range(nsteps):
        _check(L.meke_b200_step(handle, C.byref(args), _ptr(d.get("del2")), C.c_void_p(st.cuda_stream)))
    return handle


def destroy_handle(handle: int) -> None:
    lib().meke_b200_destroy(handle)
