"""Horizontal domain decomposition of the Redi step across ranks.

The Redi stencil is purely lateral-nearest-neighbour: Phase A (a face reads the
two columns either side of it) and Phase B (a cell reads its four neighbours'
columns) never reach further than one column, and there are no corner terms
(redi/ocean_redi.F90:694-812, 1148-1180). A global domain split into px x py
tiles therefore needs exactly one exchange per step: the one-column halo of h
and of every tracer, before Phase A. After it, every physical cell of a tile
sees the same inputs as in the undivided domain and gets bit-identical
results. Walls apply only on the global edges; tile edges are open.

Exchange: torch.distributed point-to-point (`batch_isend_irecv`), NCCL over
NVLink/NVSwitch on GPUs, gloo on CPU (tests). Each side packs its first/last
physical column (or row) of every field, (nz, ny) or (nz, nx) doubles, into one
contiguous buffer per neighbour; the receiver writes it into its ghost column.
On the GPU one library launch (`redi_b200_halo_copy`) packs all fields for a
neighbour and one unpacks them; CPU tensors (the gloo tests) are copied slice by
slice.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Optional

import numpy as np


def factor_tiles(world: int):
    """px x py with px * py = world, as square as possible, px >= py."""
    py = int(math.isqrt(world))
    while world % py:
        py -= 1
    return world // py, py


@dataclass
class Tiling:
    world: int
    rank: int
    px: int
    py: int

    @property
    def tx(self) -> int:
        return self.rank % self.px

    @property
    def ty(self) -> int:
        return self.rank // self.px

    def neighbour(self, dx: int, dy: int) -> Optional[int]:
        x, y = self.tx + dx, self.ty + dy
        if 0 <= x < self.px and 0 <= y < self.py:
            return y * self.px + x
        return None

    @classmethod
    def for_world(cls, world: int, rank: int, p=None) -> "Tiling":
        px, py = factor_tiles(world)
        return cls(world, rank, px, py)

    def walls(self):
        """(west, east, south, north): walls only where the tile touches the global edge."""
        return (int(self.tx == 0), int(self.tx == self.px - 1), int(self.ty == 0), int(self.ty == self.py - 1))

    def local_problem(self, p, seed_offset: int = 0):
        """This rank's tile for weak scaling: a problem of p's shape generated with a rank-specific seed.

        The tile edges are opened; the ghost columns are filled by the first exchange. Face masks on
        tile edges are made consistent between neighbours by `HaloExchange.setup_masks`.
        """
        from . import inputs

        if self.world == 1:
            return p
        q = inputs.make_problem(p.nx_phys, p.ny_phys, p.nz, n_seamounts=p.meta.get("n_seamounts", 6),
                                land_fraction=p.meta.get("land_fraction_target", 0.15),
                                n_passive=p.meta.get("n_passive", 0),
                                seed=p.meta.get("seed", 0) + 1000 * (self.rank + 1) + seed_offset,
                                nghost=p.nghost, name=f"{p.name}_tile{self.rank}")
        q.walls = self.walls()
        return q


def global_split(p, tiling: Tiling):
    """Cut an undivided problem into this rank's tile (for tests: tiles of one global field).

    The tile keeps its own ghost ring copied from the global field, so the
    result equals what the exchange produces.
    """
    from .inputs import RediProblem

    g = p.nghost
    assert p.nx_phys % tiling.px == 0 and p.ny_phys % tiling.py == 0
    nxp, nyp = p.nx_phys // tiling.px, p.ny_phys // tiling.py
    i0, j0 = tiling.tx * nxp, tiling.ty * nyp  # first physical column of the tile, in global ghosted index - g
    xs = slice(i0, i0 + nxp + 2 * g)
    ys = slice(j0, j0 + nyp + 2 * g)
    xs_u = slice(i0, i0 + nxp + 2 * g + 1)
    ys_v = slice(j0, j0 + nyp + 2 * g + 1)
    c = np.ascontiguousarray
    q = RediProblem(
        name=f"{p.name}_tile{tiling.rank}", nx_phys=nxp, ny_phys=nyp, nz=p.nz, nghost=g, dt=p.dt, eos=p.eos,
        h=c(p.h[:, ys, xs]), tracers=[c(t[:, ys, xs]) for t in p.tracers], idx_temperature=p.idx_temperature,
        idx_salinity=p.idx_salinity, dy_cu=c(p.dy_cu[ys, xs_u]), dx_cv=c(p.dx_cv[ys_v, xs]),
        idxCu=c(p.idxCu[ys, xs_u]), idyCv=c(p.idyCv[ys_v, xs]), areaT=c(p.areaT[ys, xs]),
        wet_u=c(p.wet_u[ys, xs_u]), wet_v=c(p.wet_v[ys_v, xs]), khtr_u=c(p.khtr_u[ys, xs_u]),
        khtr_v=c(p.khtr_v[ys_v, xs]), walls=tiling.walls(), meta=dict(p.meta))
    # The global edge faces stay dry as in the global problem; interior tile-edge faces keep the
    # global mask values they were cut from.
    return q


class HaloExchange:
    """One-column halo exchange of h and every tracer between neighbouring tiles.

    ``fields`` are (nz, ny, nx) tensors (device or CPU) laid out like the
    Fortran arrays; ghost width ``nghost`` >= 1, of which the innermost ghost
    column/row is exchanged.
    """

    def __init__(self, tiling: Tiling, dp=None, fields: Optional[List] = None, nghost: Optional[int] = None,
                 group=None):
        import torch
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.tiling = tiling
        if fields is None:
            fields = [dp.ms.h_layer] + list(dp.ms.tracers)
            nghost = dp.grid.nghost
        self.fields = fields
        self.g = int(nghost)
        nz, ny, nx = fields[0].shape
        self.shape = (nz, ny, nx)
        nf = len(fields)
        dev = fields[0].device
        mk = lambda n: torch.empty(n, dtype=fields[0].dtype, device=dev)  # noqa: E731
        self.sides = []
        g = self.g
        # (neighbour rank, send slice, recv slice, send buffer, recv buffer, values per field,
        #  (axis, send index, recv index) for the library's pack / unpack)
        for dx, dy in ((-1, 0), (1, 0), (0, -1), (0, 1)):
            nb = tiling.neighbour(dx, dy)
            if nb is None:
                continue
            if dx == -1:
                send, recv = (slice(None), slice(None), g), (slice(None), slice(None), g - 1)
                n, lib = nz * ny, (0, g, g - 1)
            elif dx == 1:
                send, recv = (slice(None), slice(None), nx - g - 1), (slice(None), slice(None), nx - g)
                n, lib = nz * ny, (0, nx - g - 1, nx - g)
            elif dy == -1:
                send, recv = (slice(None), g, slice(None)), (slice(None), g - 1, slice(None))
                n, lib = nz * nx, (1, g, g - 1)
            else:
                send, recv = (slice(None), ny - g - 1, slice(None)), (slice(None), ny - g, slice(None))
                n, lib = nz * nx, (1, ny - g - 1, ny - g)
            self.sides.append((nb, send, recv, mk(n * nf), mk(n * nf), n, lib))

    def _lib_copy(self, fields, axis: int, index: int, buf, to_buf: bool) -> None:
        import ctypes as C

        import torch

        from . import ocean_redi as R

        L = R.lib()
        L.redi_b200_halo_copy.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                          C.c_int, C.c_void_p, C.c_int, C.c_void_p]
        nz, ny, nx = fields[0].shape
        ptrs = (C.c_void_p * len(fields))(*[t.data_ptr() for t in fields])
        R._check(L.redi_b200_halo_copy(ptrs, len(fields), nx, ny, nz, axis, index, buf.data_ptr(), int(to_buf),
                                       torch.cuda.current_stream().cuda_stream))

    def exchange(self, fields=None):
        fields = self.fields if fields is None else fields
        on_gpu = fields[0].is_cuda and all(t.is_contiguous() and t.dtype == fields[0].dtype for t in fields)
        ops = []
        for nb, send, recv, sbuf, rbuf, n, lib in self.sides:
            if on_gpu:
                self._lib_copy(fields, lib[0], lib[1], sbuf, True)
            else:
                for f, t in enumerate(fields):
                    sbuf[f * n:(f + 1) * n].view(t[send].shape).copy_(t[send])
            ops.append(self.dist.P2POp(self.dist.isend, sbuf, nb, self.group))
            ops.append(self.dist.P2POp(self.dist.irecv, rbuf, nb, self.group))
        if ops:
            for r in self.dist.batch_isend_irecv(ops):
                r.wait()
        for nb, send, recv, sbuf, rbuf, n, lib in self.sides:
            if on_gpu:
                self._lib_copy(fields, lib[0], lib[2], rbuf, False)
            else:
                for f, t in enumerate(fields):
                    t[recv].copy_(rbuf[f * n:(f + 1) * n].view(t[recv].shape))

    def setup_masks(self, dp, cell_wet) -> None:
        """Make the face masks on tile edges agree between neighbours.

        ``cell_wet`` is this tile's (ny, nx) cell wet flag (its physical cells are
        authoritative). The flags are exchanged once; each tile-edge face is then
        wet(left) * wet(right), the rule the generator uses for every other face.
        """
        import torch

        wu, wv = dp.metrics.wet_u, dp.metrics.wet_v
        nz, ny, nx = self.shape
        g = self.g
        c = torch.as_tensor(cell_wet, dtype=wu.dtype).to(wu.device).reshape(1, ny, nx).contiguous()
        self._exchange_once([c])
        c = c[0]
        t = self.tiling
        if t.neighbour(-1, 0) is not None:
            wu[:, g] = c[:, g - 1] * c[:, g]
        if t.neighbour(1, 0) is not None:
            wu[:, nx - g] = c[:, nx - g - 1] * c[:, nx - g]
        if t.neighbour(0, -1) is not None:
            wv[g, :] = c[g - 1, :] * c[g, :]
        if t.neighbour(0, 1) is not None:
            wv[ny - g, :] = c[ny - g - 1, :] * c[ny - g, :]

    def _exchange_once(self, fields) -> None:
        """Exchange fields of another depth with buffers sized for them (set-up only)."""
        import torch

        saved = self.sides
        nz = fields[0].shape[0]
        sides = []
        for nb, send, recv, sbuf, rbuf, n, lib in saved:
            m = n // self.shape[0] * nz
            mk = lambda: torch.empty(m * len(fields), dtype=fields[0].dtype, device=fields[0].device)  # noqa: E731
            sides.append((nb, send, recv, mk(), mk(), m, lib))
        self.sides = sides
        try:
            self.exchange(fields)
        finally:
            self.sides = saved

    def close(self) -> None:
        self.sides = []
