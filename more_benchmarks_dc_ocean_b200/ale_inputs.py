"""Seeded inputs for the ALE remap step.

An ``AleProblem`` holds the state ``ale_remap_step`` (ale_remap/ale_remap.F90:76-188)
reads and writes, as numpy float64 arrays in the Fortran shapes reversed:
``h_layer`` and the budgets (nz, ny, nx); ``tracers`` a list of (nz, ny, nx)
arrays (``None`` = an unallocated slot); ``u`` (nz, ny, nx+1); ``v`` (nz, ny+1, nx);
``bt_eta`` and ``bt_H_ref`` (ny, nx); ``dsig`` (nz); and the vcoord workspaces the
step fills (``total_h``, ``h_ref`` (ny, nx), ``h_old``, ``target_h`` (nz, ny, nx)).
``method`` is the reference's remap code (1 PCM, 2 PLM, 3 PPM), ``conserve_ke``
the KE-rescale switch, ``idx_temperature`` / ``idx_salinity`` 0-based slots.

``reference_ic`` is the reference driver's state (ale_remap/drivers/cpp_main.cu:122-182,
itself a transcription of ale_bench.F90:108-157): a stretched sigma distribution,
bathymetry with vanished-layer columns, a free surface, layers perturbed by the
h-drift percentage and renormalised to the column depth, stratified T and S, and
smooth face velocities. Its default size is the reference's benchmark, 473 x 297
points with 3 ghost cells (arrays 479 x 303), 30 layers, h-drift 25 %.

``random_case`` draws uneven layers with vanished layers, zero target layers,
passive tracers and random velocities, with any of the switches overridden.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

REMAP_PCM, REMAP_PLM, REMAP_PPM, REMAP_PPM_H4, REMAP_PQM = 1, 2, 3, 4, 5
STATE = ("h_layer", "u", "v", "mass_budget", "heat_budget", "salt_budget", "bt_eta")
WORKSPACES = ("total_h", "h_ref", "h_old", "target_h")


@dataclass
class AleProblem:
    name: str
    nx: int
    ny: int
    nz: int
    h_layer: np.ndarray
    tracers: List[Optional[np.ndarray]]
    u: Optional[np.ndarray]
    v: Optional[np.ndarray]
    mass_budget: np.ndarray
    heat_budget: np.ndarray
    salt_budget: np.ndarray
    bt_eta: np.ndarray
    bt_H_ref: np.ndarray
    dsig: np.ndarray
    method: int = REMAP_PPM
    conserve_ke: bool = False
    idx_temperature: int = 0
    idx_salinity: int = 1
    total_h: np.ndarray = field(default=None)
    h_ref: np.ndarray = field(default=None)
    h_old: np.ndarray = field(default=None)
    target_h: np.ndarray = field(default=None)

    def __post_init__(self):
        n2, n3 = (self.ny, self.nx), (self.nz, self.ny, self.nx)
        for k, shape in (("total_h", n2), ("h_ref", n2), ("h_old", n3), ("target_h", n3)):
            if getattr(self, k) is None:
                setattr(self, k, np.zeros(shape))

    def copy(self) -> "AleProblem":
        c = lambda a: None if a is None else a.copy()  # noqa: E731
        return AleProblem(self.name, self.nx, self.ny, self.nz, self.h_layer.copy(), [c(t) for t in self.tracers],
                          c(self.u), c(self.v), self.mass_budget.copy(), self.heat_budget.copy(),
                          self.salt_budget.copy(), self.bt_eta.copy(), self.bt_H_ref.copy(), self.dsig.copy(),
                          self.method, self.conserve_ke, self.idx_temperature, self.idx_salinity,
                          self.total_h.copy(), self.h_ref.copy(), self.h_old.copy(), self.target_h.copy())

    def arrays(self):
        """Every array the step writes, by name (tracers as tracer0, tracer1, ...)."""
        out = {k: getattr(self, k) for k in STATE + WORKSPACES if getattr(self, k) is not None}
        for n, t in enumerate(self.tracers):
            if t is not None:
                out[f"tracer{n}"] = t
        return out


def reference_ic(nxp: int = 473, nyp: int = 297, nz: int = 30, nghost: int = 3, drift_pct: int = 25) -> AleProblem:
    """The reference driver's pristine state on an (nxp+2*nghost) x (nyp+2*nghost) x nz grid."""
    nx, ny = nxp + 2 * nghost, nyp + 2 * nghost
    k1 = np.arange(1, nz + 1, dtype=np.float64)
    dsig = 1.0 + 3.0 * (k1 - 1.0) / float(max(1, nz - 1))
    dsum = 0.0
    for d in dsig:  # in order, as Fortran's sum() over the elements
        dsum += d
    dsig = dsig / dsum
    i = np.arange(1, nx + 1, dtype=np.float64)[None, :]
    j = np.arange(1, ny + 1, dtype=np.float64)[:, None]
    hbed = 15.0 + 4485.0 * np.abs(np.sin(0.013 * i) * np.cos(0.017 * j))
    ii, jj = np.meshgrid(np.arange(1, nx + 1), np.arange(1, ny + 1))
    hbed = np.where((ii + jj) % 97 == 0, 3.0, hbed)
    eta = 0.4 * np.sin(0.05 * i + 0.03 * j)
    h = np.empty((nz, ny, nx))
    for k in range(1, nz + 1):
        pert = (0.01 * drift_pct) * np.sin(3.0 * k + 0.02 * i + 0.03 * j)
        h[k - 1] = (hbed + eta) * dsig[k - 1] * (1.0 + pert)
    csum = np.zeros((ny, nx))
    for k in range(nz):
        csum = csum + h[k]
    h = h * (hbed + eta) / csum
    T = np.empty_like(h)
    S = np.empty_like(h)
    for k in range(1, nz + 1):
        cT = 2.0 + 12.0 * np.exp(-(nz - k) / 6.0) + 0.5 * np.sin(0.02 * i)
        cS = 34.5 + 0.8 * k / nz
        T[k - 1] = h[k - 1] * cT
        S[k - 1] = h[k - 1] * cS
    iu = np.arange(1, nx + 2, dtype=np.float64)[None, :]
    jv = np.arange(1, ny + 2, dtype=np.float64)[:, None]
    u = np.empty((nz, ny, nx + 1))
    v = np.empty((nz, ny + 1, nx))
    for k in range(1, nz + 1):
        u[k - 1] = 0.3 * np.sin(0.01 * iu) * np.cos(0.02 * j) * (1.0 + 0.1 * k)
        v[k - 1] = 0.2 * np.cos(0.015 * i) * np.sin(0.018 * jv) * (1.0 - 0.05 * k)
    z3 = lambda: np.zeros((nz, ny, nx))  # noqa: E731
    return AleProblem(f"reference_ic_{nx}x{ny}x{nz}_drift{drift_pct}", nx, ny, nz, np.ascontiguousarray(h),
                      [np.ascontiguousarray(T), np.ascontiguousarray(S)], u, v, z3(), z3(), z3(),
                      np.ascontiguousarray(eta * np.ones((ny, nx))), np.ascontiguousarray(hbed), dsig)


def random_case(nx: int, ny: int, nz: int, seed: int, name: str = "", n_passive: int = 1, vanished: float = 0.15,
                zero_targets: int = 1, method: int = REMAP_PPM, conserve_ke: bool = False, faces: bool = True,
                budgets_nonzero: bool = True) -> AleProblem:
    """Uneven layers (some vanished), zero-thickness target layers, passive tracers, random velocities."""
    r = np.random.default_rng(seed)
    depth = r.uniform(5.0, 4000.0, (ny, nx))
    depth[r.random((ny, nx)) < 0.05] = 2.0  # shallow columns: every layer below H_FLOOR-scale thicknesses
    h = depth[None] / nz * r.uniform(0.2, 1.8, (nz, ny, nx))
    h[r.random((nz, ny, nx)) < vanished] = 0.0
    h[r.random((nz, ny, nx)) < 0.03] = r.uniform(0.0, 3.0e-4)  # straddling H_FLOOR
    eta = r.uniform(-1.0, 1.0, (ny, nx))
    H_ref = r.uniform(0.0, 4000.0, (ny, nx))
    dsig = r.uniform(0.2, 2.0, nz)
    if zero_targets and nz > 3:
        dsig[r.choice(nz, size=min(zero_targets, nz - 2), replace=False)] = 0.0
    dsig = dsig / dsig.sum()
    tr = [h * r.uniform(-2.0, 30.0, (nz, ny, nx)), h * r.uniform(30.0, 37.0, (nz, ny, nx))]
    tr += [h * r.standard_normal((nz, ny, nx)) for _ in range(n_passive)]
    u = r.standard_normal((nz, ny, nx + 1)) if faces else None
    v = r.standard_normal((nz, ny + 1, nx)) if faces else None
    b = (lambda: r.standard_normal((nz, ny, nx))) if budgets_nonzero else (lambda: np.zeros((nz, ny, nx)))
    return AleProblem(name or f"random_{nx}x{ny}x{nz}_s{seed}", nx, ny, nz, h, tr, u, v, b(), b(), b(), eta, H_ref,
                      dsig, method=method, conserve_ke=conserve_ke)
