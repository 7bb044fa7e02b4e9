"""Seeded synthetic inputs for the Redi neutral-diffusion step.

The reference publishes no dataset for this path; every workload is generated
here from a seed, deterministically, with the shapes and value distributions of
the benchmark configurations:

* ``config0``  128x96x25, T and S, 6 seamounts, ~15 % land (CPU-runnable case)
* ``config1``  1440x1080x75, T and S, 40 seamounts, ~30 % land (production size)
* ``config3``  720x576x50, T, S and 32 passive tracers
* ``config4``  64 uneven regional domains, T, S and 4 passive tracers each
* ``reference_ic``  the reference driver's own initial condition
  (redi/drivers/dc_main.F90:172-206: 473x297x30, nghost=3, uniform h, a tilted
  T/S front, dt=900 s, khtr=100 m^2/s, alpha_T=1.7e-4).

Array layout. Every field is stored exactly as the reference's Fortran arrays
are laid out in memory (column-major, i fastest). A numpy array therefore has
the Fortran shape reversed: a tracer ``hTr(nx, ny, nz)`` is a C-contiguous
``(nz, ny, nx)`` array, a u-face field ``(nx+1, ny)`` is ``(ny, nx+1)``, and a
u-face coefficient ``uPoL(nx+1, ny, ns)`` is ``(ns, ny, nx+1)``. Native
vertical index k=0 is the bed and k=nz-1 the surface
(redi/multilayer_cgrid_state.F90:24).

Generators (one ``numpy.random.SeedSequence([seed, field_id])`` stream per
field, so fields are independent of one another and of generation order):

* grid: dx = dy = 10 km; dy_cu = dx_cv = 1e4 m, idxCu = idyCv = 1e-4 1/m,
  areaT = 1e8 m^2; all four physical edges are no-normal-flow walls.
* bathymetry: D = 4000 - sum_m A_m exp(-|r - c_m|^2 / (2 sigma_m^2)) with
  centres uniform over the physical domain, A_m ~ U(4500, 6500) m and
  sigma_m = s * U(0.5, 1.5) * min(Lx, Ly); the common scale s is bisected at the
  fixed seed until the land fraction (D < 50 m) of the physical cells hits the
  target. wet = D >= 50 m; wet_u(i,j) = wet(i-1,j) * wet(i,j) (Fortran
  indices), wet_v likewise; the domain-edge faces are dry.
* layers: h_k = max(D, 0) / nz * (1 + 0.2 U(-1, 1)), floored at 1e-3 m.
* T = 2 + 23 exp(-z/800) + 0.5 sin(2 pi x/Lx) cos(2 pi y/Ly) + N(0, 0.05) degC,
  S = 34.5 + z/4000 + N(0, 0.01) psu, z the depth of the layer centre.
  Passive tracers: N(0, 1) white noise box-filtered over 5x5 cells per layer,
  times exp(-z/500). Stored thickness-weighted (hTr = tracer * h).
* EOS: linear, rho0 = 1035, alpha_T = 2e-4, beta_S = 7.6e-4, T_ref = 10,
  S_ref = 35. khtr = 1000 m^2/s on every face (the per-face ``khtr_*_ext`` path
  that the reference exercises), dt = 1800 s.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

# Field ids for the per-field random streams.
_F_SEAMOUNTS, _F_LAYERS, _F_TNOISE, _F_SNOISE, _F_PASSIVE0 = 1, 2, 3, 4, 100


@dataclass
class Eos:
    """ocean_eos_t (redi/ocean_eos.F90:239-278): the variant (1 LINEAR, 2 WRIGHT_97,
    4 ROQUET_SPV, the reference's codes) and the linear branch's coefficients."""

    rho0: float = 1035.0
    T_ref: float = 10.0
    S_ref: float = 35.0
    alpha_T: float = 1.7e-4
    beta_S: float = 7.6e-4
    variant: int = 1


@dataclass
class RediProblem:
    """One Redi domain: grid, metrics, EOS, state and diffusivity.

    Mirrors the reference's stub types: ``hgrid_t`` (redi/grid.F90:17-25),
    ``ocean_metrics_t`` (redi/ocean_metrics.F90:14-22),
    ``multilayer_cgrid_state_t`` (redi/multilayer_cgrid_state.F90:18-28) and the
    per-face ``khtr_u_ext``/``khtr_v_ext`` arguments of ``redi_apply_flux``.
    """

    name: str
    nx_phys: int
    ny_phys: int
    nz: int
    nghost: int
    dt: float
    eos: Eos
    h: np.ndarray              # (nz, ny, nx) layer thickness, m
    tracers: List[np.ndarray]  # each (nz, ny, nx) thickness-weighted tracer
    idx_temperature: int       # 0-based index into tracers
    idx_salinity: int
    dy_cu: np.ndarray          # (ny, nx+1)
    dx_cv: np.ndarray          # (ny+1, nx)
    idxCu: np.ndarray          # (ny, nx+1)
    idyCv: np.ndarray          # (ny+1, nx)
    areaT: np.ndarray          # (ny, nx)
    wet_u: np.ndarray          # (ny, nx+1)
    wet_v: np.ndarray          # (ny+1, nx)
    khtr_u: np.ndarray         # (ny, nx+1)
    khtr_v: np.ndarray         # (ny+1, nx)
    walls: tuple = (1, 1, 1, 1)  # west, east, south, north: 1 = no-normal-flow wall
    meta: dict = field(default_factory=dict)
    wet: Optional[np.ndarray] = None  # (ny, nx) cell wet flag (1 = ocean), where known

    @property
    def nx(self) -> int:
        return self.nx_phys + 2 * self.nghost

    @property
    def ny(self) -> int:
        return self.ny_phys + 2 * self.nghost

    @property
    def ns(self) -> int:
        return 2 * self.nz + 2

    @property
    def ntr(self) -> int:
        return len(self.tracers)

    @property
    def ncell(self) -> int:
        return self.nx * self.ny * self.nz

    def copy(self) -> "RediProblem":
        p = RediProblem(**{k: getattr(self, k) for k in self.__dataclass_fields__})
        p.h = self.h.copy()
        p.tracers = [t.copy() for t in self.tracers]
        p.meta = dict(self.meta)
        return p


def _rng(seed: int, field_id: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(np.random.SeedSequence([seed, field_id])))


def _cell_centres(nphys: int, nghost: int, d: float) -> np.ndarray:
    n = nphys + 2 * nghost
    return (np.arange(n, dtype=np.float64) - nghost + 0.5) * d


def _bathymetry(nxp, nyp, nghost, dx, n_seamounts, land_target, seed, depth=4000.0):
    """Seamount field calibrated to a land fraction; returns (D (ny,nx), scale)."""
    rng = _rng(seed, _F_SEAMOUNTS)
    lx, ly = nxp * dx, nyp * dx
    cx = rng.uniform(0.0, lx, n_seamounts)
    cy = rng.uniform(0.0, ly, n_seamounts)
    amp = rng.uniform(4500.0, 6500.0, n_seamounts)
    width = rng.uniform(0.5, 1.5, n_seamounts) * min(lx, ly)
    x = _cell_centres(nxp, nghost, dx)
    y = _cell_centres(nyp, nghost, dx)

    def field_at(xs, ys, s):
        d = np.full((ys.size, xs.size), depth)
        for m in range(n_seamounts):
            sig = s * width[m]
            gx = np.exp(-((xs - cx[m]) ** 2) / (2.0 * sig * sig))
            gy = np.exp(-((ys - cy[m]) ** 2) / (2.0 * sig * sig))
            d -= amp[m] * np.outer(gy, gx)
        return d

    # Bisect the width scale on a subsampled copy of the physical grid.
    step = max(1, min(nxp, nyp) // 128)
    xs = x[nghost:nghost + nxp:step]
    ys = y[nghost:nghost + nyp:step]
    lo, hi = 1e-4, 2.0
    s = 0.5 * (lo + hi)
    if land_target > 0.0:
        for _ in range(48):
            s = 0.5 * (lo + hi)
            frac = float(np.mean(field_at(xs, ys, s) < 50.0))
            if frac < land_target:
                lo = s
            else:
                hi = s
    else:
        s = 0.0
    d = field_at(x, y, s) if s > 0.0 else np.full((y.size, x.size), depth)
    return d, s


def _box5(a: np.ndarray) -> np.ndarray:
    """5x5 moving average over the last two axes with edge replication."""
    p = np.pad(a, [(0, 0), (2, 2), (2, 2)], mode="edge")
    ny, nx = a.shape[1], a.shape[2]
    r = p[:, 0:ny] + p[:, 1:ny + 1]  # separable running sums over contiguous slabs
    for o in (2, 3, 4):
        r += p[:, o:ny + o]
    s = r[:, :, 0:nx] + r[:, :, 1:nx + 1]
    for o in (2, 3, 4):
        s += r[:, :, o:nx + o]
    s /= 25.0
    return s


def make_problem(nx_phys: int, ny_phys: int, nz: int, *, n_seamounts: int = 6, land_fraction: float = 0.15,
                 n_passive: int = 0, seed: int = 20261203, nghost: int = 2, dx: float = 1.0e4,
                 dt: float = 1800.0, khtr: float = 1000.0, name: Optional[str] = None) -> RediProblem:
    """Generate one seeded domain with the benchmark's distributions."""
    nx, ny = nx_phys + 2 * nghost, ny_phys + 2 * nghost
    depth, scale = _bathymetry(nx_phys, ny_phys, nghost, dx, n_seamounts, land_fraction, seed)
    wet = depth >= 50.0

    r_layers = _rng(seed, _F_LAYERS)
    dpos = np.maximum(depth, 0.0)
    h = (dpos / nz)[None, :, :] * (1.0 + 0.2 * r_layers.uniform(-1.0, 1.0, (nz, ny, nx)))
    np.maximum(h, 1.0e-3, out=h)

    # Depth of layer centres: native k=0 is the bed, so accumulate from the top.
    above = np.cumsum(h[::-1], axis=0)[::-1] - h  # thickness of the layers above k
    z = above + 0.5 * h
    del above

    lx, ly = nx_phys * dx, ny_phys * dx
    x = _cell_centres(nx_phys, nghost, dx)
    y = _cell_centres(ny_phys, nghost, dx)
    horiz = 0.5 * np.outer(np.cos(2.0 * math.pi * y / ly), np.sin(2.0 * math.pi * x / lx))

    t = 2.0 + 23.0 * np.exp(-z / 800.0)
    t += horiz[None, :, :]
    t += _rng(seed, _F_TNOISE).normal(0.0, 0.05, (nz, ny, nx))
    t *= h
    s = 34.5 + z / 4000.0
    s += _rng(seed, _F_SNOISE).normal(0.0, 0.01, (nz, ny, nx))
    s *= h
    tracers = [t, s]
    if n_passive:
        decay = np.exp(-z / 500.0)
        for m in range(n_passive):
            noise = _rng(seed, _F_PASSIVE0 + m).normal(0.0, 1.0, (nz, ny, nx))
            tr = _box5(noise)
            tr *= decay
            tr *= h
            tracers.append(np.ascontiguousarray(tr))
        del decay
    del z

    wet_u = np.zeros((ny, nx + 1))
    wet_u[:, 1:nx] = (wet[:, :-1] & wet[:, 1:]).astype(np.float64)
    wet_v = np.zeros((ny + 1, nx))
    wet_v[1:ny, :] = (wet[:-1, :] & wet[1:, :]).astype(np.float64)

    return RediProblem(
        name=name or f"{nx_phys}x{ny_phys}x{nz}",
        nx_phys=nx_phys, ny_phys=ny_phys, nz=nz, nghost=nghost, dt=dt,
        eos=Eos(rho0=1035.0, T_ref=10.0, S_ref=35.0, alpha_T=2.0e-4, beta_S=7.6e-4),
        h=h, tracers=tracers, idx_temperature=0, idx_salinity=1,
        dy_cu=np.full((ny, nx + 1), dx), dx_cv=np.full((ny + 1, nx), dx),
        idxCu=np.full((ny, nx + 1), 1.0 / dx), idyCv=np.full((ny + 1, nx), 1.0 / dx),
        areaT=np.full((ny, nx), dx * dx),
        wet_u=wet_u, wet_v=wet_v,
        khtr_u=np.full((ny, nx + 1), khtr), khtr_v=np.full((ny + 1, nx), khtr),
        wet=wet.astype(np.float64),
        meta={"seed": seed, "n_seamounts": n_seamounts, "land_fraction_target": land_fraction,
              "land_fraction": float(1.0 - wet[nghost:nghost + ny_phys, nghost:nghost + nx_phys].mean()),
              "seamount_scale": scale, "n_passive": n_passive},
    )


def config0(seed: int = 20261203) -> RediProblem:
    """Plain FP64 step at 128x96x25, T and S (the CPU-runnable case)."""
    return make_problem(128, 96, 25, n_seamounts=6, land_fraction=0.15, seed=seed, name="config0_128x96x25")


def config1(seed: int = 20261203) -> RediProblem:
    """Production size 1440x1080x75, T and S, 40 seamounts, ~30 % land."""
    return make_problem(1440, 1080, 75, n_seamounts=40, land_fraction=0.30, seed=seed,
                        name="config1_1440x1080x75")


def config3(seed: int = 20261203) -> RediProblem:
    """720x576x50 with T, S and 32 passive tracers."""
    return make_problem(720, 576, 50, n_seamounts=40, land_fraction=0.30, n_passive=32, seed=seed,
                        name="config3_720x576x50_34tr")


def config4_shapes(seed: int = 20261203, n_domains: int = 64):
    """(nx_phys, ny_phys, nz) of the uneven-domain batch: nx, ny log-uniform in [64, 512]."""
    rng = _rng(seed, 7)
    nxs = np.exp(rng.uniform(math.log(64), math.log(512), n_domains)).round().astype(int)
    nys = np.exp(rng.uniform(math.log(64), math.log(512), n_domains)).round().astype(int)
    nzs = rng.choice([25, 50, 75], n_domains)
    return [(int(a), int(b), int(c)) for a, b, c in zip(nxs, nys, nzs)]


def config4_domain(seed: int, d: int, shape) -> RediProblem:
    """Domain d of the uneven-domain batch: seeded as config 0 with its own seamounts and mask."""
    a, b, c = shape
    return make_problem(a, b, c, n_seamounts=6, land_fraction=0.15, n_passive=4, seed=seed + 1 + d,
                        name=f"config4_d{d}_{a}x{b}x{c}")


def _config4_job(job):
    return config4_domain(*job)


def config4(seed: int = 20261203, n_domains: int = 64, shapes=None, workers: int = 1) -> List[RediProblem]:
    """Uneven-domain batch: 64 domains, T, S and 4 passive tracers each.

    ``workers`` > 1 generates the domains in a pool of spawned processes (the
    result does not depend on it).
    """
    shapes = shapes or config4_shapes(seed, n_domains)
    jobs = [(seed, d, s) for d, s in enumerate(shapes)]
    if workers <= 1:
        return [_config4_job(j) for j in jobs]
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor

    # largest first so the pool's tail is short; results returned in domain order
    order = sorted(range(len(jobs)), key=lambda i: -jobs[i][2][0] * jobs[i][2][1] * jobs[i][2][2])
    out: List[Optional[RediProblem]] = [None] * len(jobs)
    with ProcessPoolExecutor(workers, mp_context=mp.get_context("spawn")) as ex:
        for i, p in zip(order, ex.map(_config4_job, [jobs[i] for i in order])):
            out[i] = p
    return out


def reference_ic(nx_phys: int = 473, ny_phys: int = 297, nz: int = 30) -> RediProblem:
    """The reference driver's initial condition (redi/drivers/dc_main.F90:60-81, 172-206).

    Uniform h = 4000/nz, T = 2 + 16 exp(-z/800) + 3 fx + 3 fy,
    S = 34.5 + 0.7 (1 - exp(-z/1500)) - 0.2 fx, all faces wet, 0.1-degree-like
    metrics (dy_cu = 11100, dx_cv = 8000), khtr_ext = 100 m^2/s, dt = 900 s,
    nghost = 3, default EOS (alpha_T = 1.7e-4).
    """
    nghost = 3
    nx, ny = nx_phys + 2 * nghost, ny_phys + 2 * nghost
    hh = 4000.0 / nz
    kk = np.arange(1, nz + 1, dtype=np.float64)           # Fortran kk = 1..nz (bottom-up)
    zz = (nz - kk + 0.5) * hh                             # dc_main.F90:193
    fx = np.arange(nx, dtype=np.float64) / (nx - 1)
    fy = np.arange(ny, dtype=np.float64) / (ny - 1)
    e800 = np.exp(-zz / 800.0)
    e1500 = np.exp(-zz / 1500.0)
    tt = (2.0 + 16.0 * e800)[:, None, None] + 3.0 * fx[None, None, :] + 3.0 * fy[None, :, None]
    ss = np.broadcast_to((34.5 + 0.7 * (1.0 - e1500))[:, None, None] - 0.2 * fx[None, None, :], (nz, ny, nx))
    h = np.full((nz, ny, nx), hh)
    return RediProblem(
        name=f"reference_ic_{nx_phys}x{ny_phys}x{nz}", nx_phys=nx_phys, ny_phys=ny_phys, nz=nz, nghost=nghost,
        dt=900.0, eos=Eos(), h=h, tracers=[np.ascontiguousarray(tt * hh), np.ascontiguousarray(ss * hh)], idx_temperature=0, idx_salinity=1,
        dy_cu=np.full((ny, nx + 1), 11100.0), dx_cv=np.full((ny + 1, nx), 8000.0),
        idxCu=np.full((ny, nx + 1), 1.0 / 8000.0), idyCv=np.full((ny + 1, nx), 1.0 / 11100.0),
        areaT=np.full((ny, nx), 8000.0 * 11100.0),
        wet_u=np.ones((ny, nx + 1)), wet_v=np.ones((ny + 1, nx)),
        khtr_u=np.full((ny, nx + 1), 100.0), khtr_v=np.full((ny + 1, nx), 100.0),
        wet=np.ones((ny, nx)), meta={"source": "redi/drivers/dc_main.F90:172-206"},
    )
