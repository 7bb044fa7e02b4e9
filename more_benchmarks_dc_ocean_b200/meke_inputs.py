"""Seeded inputs for the MEKE step.

A ``MekeProblem`` holds every array of the reference's argument block
(meke/meke_args.h:38-52) as numpy float64 in the Fortran shapes reversed:
cell fields (ny, nx), u faces (ny, nx+1), v faces (ny+1, nx), layers
(nz, ny, nx); plus ``del2`` (ocean_meke_t%del2) and the configuration scalars
under their MekeArgs names (``kh_bg`` is ocean_meke_t%kh).

``reference_ic`` is the reference driver's state (meke/drivers/cpp_main.cu:133-186,
itself a transcription of meke_bench.F90:106-126 and 336-363): uniform 8 km
metrics, a stratified column, a Gaussian GM source and eddy energy, a
beta-plane |f|, and the one configuration that turns MEKE on
(gabight_sph_meke_v100: gmcoeff 0.9, khcoeff 1, cdrag 2.5e-3, kh 100, the
ocean_meke_t defaults otherwise). Its default size is the reference's
benchmark, 473 x 297 points with 3 ghost cells (arrays 479 x 303) and 30
layers.

``random_case`` draws non-uniform metrics, layers with vanished and land
columns, and signed energies, with any configuration scalars overridden, so
that every branch of the step can be made live.
"""

from __future__ import annotations

import copy
from dataclasses import dataclass, field
from typing import Dict

import numpy as np

CELL = ("meke", "kh_diff", "le", "ku", "i_mass", "depth_tot", "bottom_fac2", "barotr_fac2", "src", "mass_ws",
        "rd_ws", "ke_diss_ws", "del2", "u_bbl2", "f_centre", "gm_src", "ke_diss_ext", "areaT", "iareaT", "idxT",
        "idyT")
UFACE = ("uflux", "sn_u_ws", "dy_cu", "idxCu")
VFACE = ("vflux", "sn_v_ws", "dx_cv", "idyCv")
LAYER = ("h_layer", "rho_layer")
# the arrays a step writes (ocean_meke_t members)
OUTPUTS = ("meke", "kh_diff", "le", "ku", "i_mass", "depth_tot", "bottom_fac2", "barotr_fac2", "src", "uflux",
           "vflux", "mass_ws", "rd_ws", "sn_u_ws", "sn_v_ws", "ke_diss_ws", "del2")
SCALARS = ("dt", "dtscale", "cd_scale", "cb", "ct", "min_gamma2", "cdrag", "uscale", "a_deform", "a_rhines",
           "a_eady", "a_frict", "a_grid", "bgsrc", "gmcoeff", "frcoeff", "damping", "kh_bg", "k4", "khmeke_fac",
           "khcoeff", "visc_coeff_ku", "rho0", "backscatter")

# ocean_meke_t defaults (meke/meke_state.F90:52-80) as MekeArgs scalars, and ocean_gm_t%rho0
DEFAULTS = dict(dtscale=1.0, cd_scale=0.0, cb=25.0, ct=50.0, min_gamma2=1.0e-4, cdrag=2.5e-3, uscale=0.0,
                a_deform=0.0, a_rhines=0.0, a_eady=0.0, a_frict=0.0, a_grid=0.0, bgsrc=0.0, gmcoeff=-1.0,
                frcoeff=-1.0, damping=0.0, kh_bg=-1.0, k4=-1.0, khmeke_fac=0.0, khcoeff=1.0, visc_coeff_ku=0.0,
                rho0=1035.0, backscatter=0)
# gabight_sph_meke_v100: enable, gmcoeff 0.9, khcoeff 1.0, cdrag 2.5e-3, kh 100
GABIGHT = dict(DEFAULTS, gmcoeff=0.9, khcoeff=1.0, cdrag=2.5e-3, kh_bg=100.0)


@dataclass
class MekeProblem:
    name: str
    nx: int
    ny: int
    nz: int
    arrays: Dict[str, np.ndarray]
    config: Dict[str, float] = field(default_factory=dict)

    @property
    def cells(self) -> int:
        return self.nx * self.ny

    def copy(self) -> "MekeProblem":
        return MekeProblem(self.name, self.nx, self.ny, self.nz, {k: v.copy() for k, v in self.arrays.items()},
                           copy.deepcopy(self.config))


def _blank(nx: int, ny: int, nz: int) -> Dict[str, np.ndarray]:
    a = {k: np.zeros((ny, nx)) for k in CELL}
    a.update({k: np.zeros((ny, nx + 1)) for k in UFACE})
    a.update({k: np.zeros((ny + 1, nx)) for k in VFACE})
    a.update({k: np.zeros((nz, ny, nx)) for k in LAYER})
    return a


def reference_ic(nxp: int = 473, nyp: int = 297, nz: int = 30, nghost: int = 3) -> MekeProblem:
    """The reference driver's initial state on an (nxp+2*nghost) x (nyp+2*nghost) x nz grid."""
    nx, ny = nxp + 2 * nghost, nyp + 2 * nghost
    dxm = dym = 8000.0
    a = _blank(nx, ny, nz)
    a["areaT"][:] = dxm * dym
    a["iareaT"][:] = 1.0 / (dxm * dym)
    a["idxT"][:] = 1.0 / dxm
    a["idyT"][:] = 1.0 / dym
    a["dy_cu"][:] = dym
    a["idxCu"][:] = 1.0 / dxm
    a["dx_cv"][:] = dxm
    a["idyCv"][:] = 1.0 / dym
    k = np.arange(1, nz + 1, dtype=np.float64)
    a["h_layer"][:] = 4000.0 / nz
    a["rho_layer"][:] = (1025.0 + 5.0 * (nz - k) / nz)[:, None, None]
    i = np.arange(1, nx + 1)
    j = np.arange(1, ny + 1)
    # C integer division of the point counts, as the reference's meke/drivers/cpp_main.cu writes them
    ga = (i - nx // 2).astype(np.float64) / max(nx // 6, 1)
    gb = (j - ny // 2).astype(np.float64) / max(ny // 6, 1)
    a["gm_src"][:] = 1.0e-2 * np.exp(-(ga[None, :] ** 2 + gb[:, None] ** 2))
    a["ke_diss_ext"][:] = -1.0e-3
    ea = (i - nx // 3).astype(np.float64) / max(nx // 8, 1)
    eb = (j - ny // 3).astype(np.float64) / max(ny // 8, 1)
    a["meke"][:] = 1.0e-3 + 1.0e-2 * np.exp(-(ea[None, :] ** 2 + eb[:, None] ** 2))
    a["f_centre"][:] = np.abs(-1.0e-4 + 2.0e-11 * (j - ny // 2).astype(np.float64) * dym)[:, None]
    return MekeProblem(f"reference_ic_{nx}x{ny}x{nz}", nx, ny, nz, a, dict(GABIGHT, dt=1800.0))


def random_case(nx: int, ny: int, nz: int, seed: int, name: str = "", land_fraction: float = 0.15,
                vanished_fraction: float = 0.1, negative_fraction: float = 0.05, **config) -> MekeProblem:
    """Non-uniform metrics, uneven layers with vanished layers and land columns, signed energies."""
    r = np.random.default_rng(seed)
    a = _blank(nx, ny, nz)
    dx = 8000.0 * r.uniform(0.6, 1.4, (ny, nx))
    dy = 8000.0 * r.uniform(0.6, 1.4, (ny, nx))
    a["areaT"][:] = dx * dy
    a["iareaT"][:] = 1.0 / a["areaT"]
    a["idxT"][:] = 1.0 / dx
    a["idyT"][:] = 1.0 / dy
    a["dy_cu"][:] = 8000.0 * r.uniform(0.6, 1.4, (ny, nx + 1))
    a["idxCu"][:] = 1.0 / (8000.0 * r.uniform(0.6, 1.4, (ny, nx + 1)))
    a["dx_cv"][:] = 8000.0 * r.uniform(0.6, 1.4, (ny + 1, nx))
    a["idyCv"][:] = 1.0 / (8000.0 * r.uniform(0.6, 1.4, (ny + 1, nx)))
    depth = r.uniform(200.0, 5000.0, (ny, nx))
    land = r.random((ny, nx)) < land_fraction
    h = depth[None] / max(nz, 1) * r.uniform(0.3, 1.7, (nz, ny, nx))
    h[r.random((nz, ny, nx)) < vanished_fraction] = 0.0
    h[:, land] = r.uniform(0.0, 1.0e-4, (nz, int(land.sum())))
    a["h_layer"][:] = h
    a["rho_layer"][:] = r.uniform(1020.0, 1030.0, (nz, ny, nx))
    e = r.uniform(0.0, 2.0e-2, (ny, nx))
    e[r.random((ny, nx)) < negative_fraction] *= -0.05
    a["meke"][:] = e
    a["kh_diff"][:] = r.uniform(0.0, 300.0, (ny, nx))
    y = np.linspace(-1.0, 1.0, ny)[:, None] + 0.01 * r.standard_normal((ny, nx))
    a["f_centre"][:] = np.abs(1.0e-4 * y)
    a["gm_src"][:] = r.uniform(0.0, 2.0e-2, (ny, nx))
    a["ke_diss_ext"][:] = -r.uniform(0.0, 2.0e-3, (ny, nx))
    a["u_bbl2"][:] = r.uniform(0.0, 4.0e-2, (ny, nx))
    # workspaces start from noise: the step must overwrite what it owns
    for k in ("le", "ku", "i_mass", "depth_tot", "bottom_fac2", "barotr_fac2", "src", "mass_ws", "rd_ws",
              "ke_diss_ws", "del2", "uflux", "vflux", "sn_u_ws", "sn_v_ws"):
        a[k][:] = r.standard_normal(a[k].shape)
    cfg = dict(GABIGHT, dt=1800.0)
    cfg.update(config)
    return MekeProblem(name or f"random_{nx}x{ny}x{nz}_s{seed}", nx, ny, nz, a, cfg)


def all_terms(**over) -> Dict[str, float]:
    """A configuration with every optional term of the step live."""
    c = dict(cd_scale=0.3, min_gamma2=2.0e-2, uscale=0.02, a_deform=1.0, a_rhines=0.15, a_eady=0.5, a_frict=0.8,
             a_grid=0.4, bgsrc=1.0e-9, frcoeff=0.5, damping=2.0e-6, khmeke_fac=0.7, backscatter=1,
             visc_coeff_ku=-0.25)
    c.update(over)
    return c
