"""Autotuner for the launch shape of the Phase-B cell update.

The cell update is tiled as a bx x by block of T-cell columns and walks each
column in vertical chunks of `chunk` layers (see csrc/redi_plain.cu). Results
are identical for every choice; speed is not: the tile sets how many
neighbouring columns and face rows a block shares through L1, the chunk sets
the L2 working set between the W, E, S and N passes against the lane
divergence at chunk edges. The tuner times every candidate on the live problem
with the library's own CUDA-event launch timing and keeps the fastest,
caching it per (GPU name, domain size class, nz, tracer count, precision) in a
JSON file (``$REDI_B200_TUNING_CACHE`` or ``~/.cache/redi_b200/tuning.json``).
"""

from __future__ import annotations

import ctypes as C
import json
import os
from typing import Iterable, Optional, Sequence, Tuple

TILES: Tuple[Tuple[int, int], ...] = ((32, 4), (64, 2), (128, 1), (32, 2), (32, 1))
CHUNKS: Tuple[int, ...] = (4, 8, 16)
# Tiles of 128 threads also run the gather with its per-layer sums in shared memory.
SMEM_TILES: Tuple[Tuple[int, int], ...] = ((32, 4), (64, 2), (128, 1))
K_CELL_UPDATE = 3


def _cache_path() -> str:
    return os.environ.get("REDI_B200_TUNING_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "redi_b200", "tuning.json"))


def _bind(L):
    L.redi_b200_set_tuning.argtypes = [C.c_int, C.c_int, C.c_int]
    L.redi_b200_get_tuning.argtypes = [C.POINTER(C.c_int)] * 3
    L.redi_b200_profile_end.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_ulonglong), C.c_int]
    return L


def get_tuning() -> Tuple[int, int, int]:
    from . import ocean_redi as R

    L = _bind(R.lib())
    bx, by, ch = C.c_int(), C.c_int(), C.c_int()
    R._check(L.redi_b200_get_tuning(C.byref(bx), C.byref(by), C.byref(ch)))
    return bx.value, by.value, ch.value


def set_tuning(bx: int, by: int, chunk: int) -> None:
    from . import ocean_redi as R

    R._check(_bind(R.lib()).redi_b200_set_tuning(int(bx), int(by), int(chunk)))


def set_tracer_group(max_group: int) -> None:
    """Largest tracer group of one face-flux launch (1, 2, 4, 8)."""
    from . import ocean_redi as R

    L = R.lib()
    L.redi_b200_set_tracer_group.argtypes = [C.c_int]
    R._check(L.redi_b200_set_tracer_group(int(max_group)))


FOLD_FP64, FOLD_MIXED, FOLD_MIXED_ORDERED = 1, 2, 4


def set_fold(enable: int = FOLD_FP64, rows: int = 2, tracers: int = 0) -> None:
    """Phase B as the fused face-flux + fold pass or the face-flux / cell-gather pair. enable is a
    mask: FOLD_FP64 (the FP64 form), FOLD_MIXED (the mixed form, in any order), FOLD_MIXED_ORDERED
    (the mixed form in the reference's order); True means FOLD_FP64. rows: cell rows per tile
    (1, 2); tracers per pass (1, 2, 4, 0 = automatic)."""
    from . import ocean_redi as R

    L = R.lib()
    L.redi_b200_set_fold.argtypes = [C.c_int, C.c_int, C.c_int]
    R._check(L.redi_b200_set_fold(int(enable), int(rows), int(tracers)))


def get_fold() -> Tuple[int, int, int]:
    """(enable mask, rows, tracers)."""
    from . import ocean_redi as R

    L = R.lib()
    L.redi_b200_get_fold.argtypes = [C.POINTER(C.c_int)] * 3
    e, r, t = C.c_int(), C.c_int(), C.c_int()
    R._check(L.redi_b200_get_fold(C.byref(e), C.byref(r), C.byref(t)))
    return e.value, r.value, t.value


def fold_shape(precision: int, nz: int, ntracers: int) -> Tuple[int, int]:
    """(rows, tracers per pass) the fused pass runs with; tracers == 0: the pair runs."""
    from . import ocean_redi as R

    L = R.lib()
    L.redi_b200_fold_shape.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    r, t = C.c_int(), C.c_int()
    R._check(L.redi_b200_fold_shape(int(precision), int(nz), int(ntracers), C.byref(r), C.byref(t)))
    return r.value, t.value


def set_gather_tracers(n: int, smem: int = 0) -> None:
    """Tracers one cell-gather launch folds (2, 4, or 8: one gather over two face-flux launches of 4,
    with shared-memory sums and 4-layer chunks) and where its per-layer sums live: 0 registers,
    1 shared memory, 2 shared memory with 8 sublayers fetched per round trip, 3 shared memory with
    batches of 4 software-pipelined (the next batch in flight while one is folded)."""
    from . import ocean_redi as R

    L = R.lib()
    L.redi_b200_set_gather_tracers.argtypes = [C.c_int, C.c_int]
    R._check(L.redi_b200_set_gather_tracers(int(n), int(smem)))


def set_sweep_form(form: int) -> None:
    """Neutral sweep form: 0 register windows, 3 / 4 / 5 both windows in a shared-memory ring of that size."""
    from . import ocean_redi as R

    L = R.lib()
    L.redi_b200_set_sweep_form.argtypes = [C.c_int]
    R._check(L.redi_b200_set_sweep_form(int(form)))


def get_sweep_form() -> int:
    from . import ocean_redi as R

    return int(R.lib().redi_b200_get_sweep_form())


def set_flux_staged(form: int) -> None:
    """Face flux form: 0 direct loads, 1 the next sublayer's reconstruction staged in shared memory
    (cp.async), 2 each column's reconstruction read through a two-layer ring in shared memory."""
    from . import ocean_redi as R

    L = R.lib()
    L.redi_b200_set_flux_staged.argtypes = [C.c_int]
    R._check(L.redi_b200_set_flux_staged(int(form)))


def get_flux_staged() -> int:
    from . import ocean_redi as R

    return int(R.lib().redi_b200_get_flux_staged())


def get_gather_tracers() -> Tuple[int, int]:
    """(tracers per gather, sums: 0 registers, 1 shared memory, 2 shared memory with 8-deep batches)."""
    from . import ocean_redi as R

    L = R.lib()
    L.redi_b200_get_gather_tracers.argtypes = [C.POINTER(C.c_int)]
    sm = C.c_int()
    n = L.redi_b200_get_gather_tracers(C.byref(sm))
    return int(n), int(sm.value)


def get_tracer_group() -> int:
    from . import ocean_redi as R

    return int(R.lib().redi_b200_get_tracer_group())


def tune_tracer_group(dp, redi, reps: int = 2, stream=None) -> dict:
    """Time redi_apply_flux for every (face-flux tracer group, tracers per gather) the tracer count
    allows; keep the fastest. Advances dp's tracers in place. Returns
    {"best": (group, gather tracers), "ms": {...: ms per apply_flux}}.
    """
    import torch

    from . import ocean_redi as R

    ntr = len(dp.ms.tracers)
    smem = get_gather_tracers()[1]
    caps = [(g, n) for g in (2, 4, 8) if g <= max(2, ntr) for n in (2, 4) if n <= g]
    if ntr > 4:
        caps.append((4, 8))  # one gather over two face-flux launches of 4
    st = torch.cuda.current_stream() if stream is None else stream
    times = {}
    for g in caps:
        set_tracer_group(g[0])
        set_gather_tracers(g[1], smem)
        R.redi_apply_flux(dp.grid, dp.metrics, redi, dp.ms, dp.dt, dp.khtr_u_ext, dp.khtr_v_ext, dp.bc, st)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(reps):
            R.redi_apply_flux(dp.grid, dp.metrics, redi, dp.ms, dp.dt, dp.khtr_u_ext, dp.khtr_v_ext, dp.bc, st)
        e1.record(st)
        torch.cuda.synchronize()
        times[g] = e0.elapsed_time(e1) / reps
    best = min(times, key=times.get)
    set_tracer_group(best[0])
    set_gather_tracers(best[1], smem)
    return {"best": best, "ms": {f"flux{g}/gather{n}": round(v, 4) for (g, n), v in times.items()}}


def _key(dp, precision: int) -> str:
    import torch

    name = torch.cuda.get_device_name(dp.ms.h_layer.device)
    cells = dp.grid.nx_total * dp.grid.ny_total
    size_class = "large" if cells >= 1 << 20 else ("medium" if cells >= 1 << 16 else "small")
    return f"{name}|{size_class}|nz{dp.ms.nz_ml}|ntr{len(dp.ms.tracers)}|p{precision}"


def load_cached(dp, precision: int = 0) -> Optional[Tuple[int, int, int]]:
    path = _cache_path()
    try:
        with open(path) as f:
            d = json.load(f)
        v = d.get(_key(dp, precision))
        return tuple(v) if v else None
    except (OSError, ValueError):
        return None


def _store(dp, precision: int, best) -> None:
    path = _cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        try:
            with open(path) as f:
                d = json.load(f)
        except (OSError, ValueError):
            d = {}
        d[_key(dp, precision)] = list(best)
        with open(path, "w") as f:
            json.dump(d, f, indent=1)
    except OSError:
        pass


def _apply(cand) -> None:
    """(bx, by, chunk[, smem]) -> the library's gather shape; the tracer count per gather is kept."""
    set_tuning(*cand[:3])
    set_gather_tracers(get_gather_tracers()[0], int(cand[3]) if len(cand) > 3 else 0)


def tune(dp, redi, candidates: Optional[Iterable[Tuple[int, ...]]] = None, reps: int = 2,
         use_cache: bool = True, stream=None) -> dict:
    """Time the cell update for every (bx, by, chunk[, smem]) candidate and keep the fastest.

    smem = 1 runs the gather with its per-layer sums in shared memory (128-thread tiles), 2 the same
    with 8 sublayers fetched per round trip, 3 with batches of 4 software-pipelined.
    Runs redi_apply_flux on ``dp`` (its tracers are advanced in place). Returns
    {"best": (bx, by, chunk, smem), "ms": {candidate: ms per launch}, "cached": bool}.
    """
    import torch

    from . import ocean_redi as R

    prec = getattr(redi, "precision", 0)
    if use_cache:
        hit = load_cached(dp, prec)
        if hit:
            _apply(hit)
            return {"best": hit, "ms": {}, "cached": True}
    L = _bind(R.lib())
    cands = list(candidates) if candidates is not None else (
        [(bx, by, c, 0) for (bx, by) in TILES for c in CHUNKS] +
        [(bx, by, c, m) for (bx, by) in SMEM_TILES for c in CHUNKS for m in (1, 2, 3)])
    R.redi_calc_coeffs(dp.grid, dp.metrics, dp.eos, redi, dp.ms, stream)
    times = {}
    for cand in cands:
        _apply(cand)
        R.redi_apply_flux(dp.grid, dp.metrics, redi, dp.ms, dp.dt, dp.khtr_u_ext, dp.khtr_v_ext, dp.bc, stream)
        torch.cuda.synchronize()
        L.redi_b200_profile_begin()
        for _ in range(reps):
            R.redi_apply_flux(dp.grid, dp.metrics, redi, dp.ms, dp.dt, dp.khtr_u_ext, dp.khtr_v_ext, dp.bc, stream)
        kt = (C.c_double * R.lib().redi_b200_kernel_count())()
        kc = (C.c_ulonglong * R.lib().redi_b200_kernel_count())()
        R._check(L.redi_b200_profile_end(kt, kc, len(kt)))
        kid = K_CELL_UPDATE
        times[cand] = kt[kid] / max(1, kc[kid])
    best = min(times, key=times.get)
    _apply(best)
    _store(dp, prec, best)
    return {"best": best, "ms": {f"{k[0]}x{k[1]}/ch{k[2]}" + ({1: "/smem", 2: "/smem/u8", 3: "/smem/pipe"}.get(k[3], "") if len(k) > 3 else ""): round(v, 4)
                                 for k, v in times.items()}, "cached": False}


# Gather tiles of the persistent multi-domain kernel: its blocks are 128 threads.
BATCH_TILES: Tuple[Tuple[int, int], ...] = ((32, 4), (16, 8))
BATCH_OCCUPANCY: Tuple[int, ...] = (4, 5, 6)
K_DOMAIN_PERSISTENT = 8


def tune_batch(batch, candidates: Optional[Iterable[Tuple[int, int, int]]] = None, reps: int = 2,
               stream=None) -> dict:
    """Time whole batch steps for every (bx, by, chunk, occupancy) candidate and keep the fastest.

    The persistent kernel runs every stage of every domain, so the candidate is
    compared on the full step (its tracers are advanced in place). Returns
    {"best": (bx, by, chunk, occupancy), "ms": {candidate: ms per step}}.
    """
    import torch

    from . import ocean_redi as R

    L = _bind(R.lib())
    cands = list(candidates) if candidates is not None else [(bx, by, c, o) for (bx, by) in BATCH_TILES
                                                             for c in CHUNKS for o in BATCH_OCCUPANCY]
    times = {}
    for cand in cands:
        batch.set_tuning(cand[:2], cand[2], cand[3] if len(cand) > 3 else 0)
        batch.step(1, stream)  # graph capture + warm-up
        torch.cuda.synchronize()
        L.redi_b200_profile_begin()
        batch.step(reps, stream)
        kt = (C.c_double * R.lib().redi_b200_kernel_count())()
        kc = (C.c_ulonglong * R.lib().redi_b200_kernel_count())()
        R._check(L.redi_b200_profile_end(kt, kc, len(kt)))
        times[cand] = kt[K_DOMAIN_PERSISTENT] / max(1, kc[K_DOMAIN_PERSISTENT])
    best = min(times, key=times.get)
    batch.set_tuning(best[:2], best[2], best[3] if len(best) > 3 else 0)
    return {"best": best, "ms": {"x".join(map(str, k[:2])) + f"/ch{k[2]}" + (f"/occ{k[3]}" if len(k) > 3 else ""):
                                 round(v, 4) for k, v in times.items()}}
