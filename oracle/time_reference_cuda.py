"""TEST INFRASTRUCTURE ONLY: the reference's own CUDA against this repository's kernels.

Times the reference's optimized launcher `redi_opt_launch` (redi/opt_kernel.cu:534-574,
compiled from the reference sources with the reference's own flags for sm_100a by
oracle/ref_build.sh into oracle/_ref/libredi_refcuda_native.so) and this repository's
export of the same symbol (libredi_b200.so) on identical device arrays, and this
repository's stream-ordered handle API (redi_b200_calc_coeffs + redi_b200_apply_flux).
Both launchers synchronise the device before returning; each call is bracketed by CUDA
events. The reference build contracts multiplies and adds into FMAs (its Makefile's
flags), so its tracers differ from the FMA-free form in the last bits: the script
reports that difference.

    python oracle/time_reference_cuda.py [--case reference_ic|config1] [--reps N]

Prints one JSON line per case. Needs a GPU and the two libraries built.
"""

from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

NATIVE = os.path.join(ROOT, "oracle", "_ref", "libredi_refcuda_native.so")


def _state(p, torch):
    dev = "cuda"
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev, torch.float64)  # noqa: E731
    ns = p.ns
    st = {"h": d(p.h), "T": d(p.tracers[0]), "S": d(p.tracers[1]), "wet_u": d(p.wet_u), "wet_v": d(p.wet_v),
          "ku_ext": d(p.khtr_u), "kv_ext": d(p.khtr_v), "dy_cu": d(p.dy_cu), "dx_cv": d(p.dx_cv),
          "idxCu": d(p.idxCu), "idyCv": d(p.idyCv), "areaT": d(p.areaT)}
    for side, (a, b) in (("u", (p.ny, p.nx + 1)), ("v", (p.ny + 1, p.nx))):
        st[side + "PoL"] = torch.zeros((ns, a, b), dtype=torch.float64, device=dev)
        st[side + "PoR"] = torch.zeros((ns, a, b), dtype=torch.float64, device=dev)
        st[side + "KoL"] = torch.ones((ns, a, b), dtype=torch.int32, device=dev)
        st[side + "KoR"] = torch.ones((ns, a, b), dtype=torch.int32, device=dev)
        st[side + "hEff"] = torch.zeros((ns - 1, a, b), dtype=torch.float64, device=dev)
    st["ku"] = torch.zeros_like(st["ku_ext"])
    st["kv"] = torch.zeros_like(st["kv_ext"])
    st["snap"] = torch.zeros_like(st["T"])
    return st


def _args(p, st):
    ci = lambda v: C.byref(C.c_int(int(v)))  # noqa: E731
    cd = lambda v: C.byref(C.c_double(float(v)))  # noqa: E731
    vp = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    e = p.eos
    ww, we, ws, wn = p.walls
    return [ci(p.nx), ci(p.ny), ci(p.nz), ci(p.ns), cd(p.dt), ci(p.nghost), ci(p.nx_phys), ci(p.ny_phys),
            ci(ww), ci(we), ci(ws), ci(wn), cd(e.rho0), cd(e.T_ref), cd(e.S_ref), cd(e.alpha_T), cd(e.beta_S),
            vp(st["h"]), vp(st["T"]), vp(st["S"]), vp(st["wet_u"]), vp(st["wet_v"]),
            vp(st["uPoL"]), vp(st["uPoR"]), vp(st["uKoL"]), vp(st["uKoR"]), vp(st["uhEff"]),
            vp(st["vPoL"]), vp(st["vPoR"]), vp(st["vKoL"]), vp(st["vKoR"]), vp(st["vhEff"]),
            vp(st["ku_ext"]), vp(st["kv_ext"]), vp(st["ku"]), vp(st["kv"]),
            vp(st["dy_cu"]), vp(st["dx_cv"]), vp(st["idxCu"]), vp(st["idyCv"]), vp(st["areaT"]), vp(st["snap"])]


def _time_calls(fn, reps, torch):
    fn()  # warm-up (first-call set-up, caches)
    fn()
    torch.cuda.synchronize()
    times = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
    return min(times), float(np.median(times))


def run(case: str, reps: int) -> dict:
    import torch

    from more_benchmarks_dc_ocean_b200 import inputs
    from more_benchmarks_dc_ocean_b200 import ocean_redi as R

    p = inputs.reference_ic() if case == "reference_ic" else getattr(inputs, case)()
    ref = C.CDLL(NATIVE)
    ours = R.lib()
    for L in (ref, ours):
        L.redi_opt_launch.restype = None
    updates = 2 * p.nx_phys * p.ny_phys * p.nz
    out = {"case": case, "grid": [p.nx_phys, p.ny_phys, p.nz], "nghost": p.nghost, "tracers": 2, "reps": reps}

    # One call each from the same initial state: how far the FMA-contracted reference is from the FMA-free form.
    s_ref, s_our = _state(p, torch), _state(p, torch)
    ref.redi_opt_launch(*_args(p, s_ref))
    ours.redi_opt_launch(*_args(p, s_our))
    torch.cuda.synchronize()
    diff = max(float(((s_ref[k] - s_our[k]).abs().max() / s_our[k].abs().max()).item()) for k in ("T", "S"))
    out["max_rel_diff_T_S_one_call"] = diff
    del s_ref, s_our
    torch.cuda.empty_cache()

    for name, L in (("reference_redi_opt_launch", ref), ("b200_redi_opt_launch", ours)):
        st = _state(p, torch)
        args = _args(p, st)
        best, med = _time_calls(lambda: L.redi_opt_launch(*args), reps, torch)
        out[name] = {"ms_min": round(best, 3), "ms_median": round(med, 3), "updates_per_s": updates / (best * 1e-3)}
        del st, args
        torch.cuda.empty_cache()

    dp = R.to_device(p)
    redi = R.make_redi(dp)
    best, med = _time_calls(lambda: R.step(dp, redi, 1), reps, torch)
    out["b200_handle_api"] = {"ms_min": round(best, 3), "ms_median": round(med, 3),
                              "updates_per_s": updates / (best * 1e-3)}
    redi.destroy()
    out["speedup_b200_vs_reference_same_launcher"] = (out["reference_redi_opt_launch"]["ms_min"] /
                                                      out["b200_redi_opt_launch"]["ms_min"])
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", action="append", choices=["reference_ic", "config0", "config1"])
    ap.add_argument("--reps", type=int, default=5)
    args = ap.parse_args()
    for case in args.case or ["reference_ic", "config1"]:
        print(json.dumps(run(case, args.reps)), flush=True)


if __name__ == "__main__":
    main()
