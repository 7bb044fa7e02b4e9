"""Generate the golden vectors that pin the MEKE CPU oracle.

Runs the reference's own CUDA launcher `meke_cuda_launch` (meke/meke_kernel.cu,
mode 0: the faithful 16-kernel form), built from the reference sources by
oracle/ref_build.sh into oracle/_ref/libmeke_refcuda.so with FMA contraction
off, on small seeded cases, and stores inputs and the outputs after every step
as compressed .npz fixtures beside this script (tests/test_meke_cpu.py checks
the oracle against them on any machine).

The cases keep kh >= 0 and k4 < 0: the reference's CUDA launchers run the
lateral step unconditionally and have no biharmonic block, so only there do
they compute meke_step_ext (meke/meke.F90:60-131).

It also records, in golden_report_meke.json: whether the reference's modes 1
(fused), 2 (graph) and `meke_opt_launch` (meke/opt_kernel.cu) agree with mode 0
on each case (meke_opt_launch is exact only for khmeke_fac == 0, its
documented caveat), and the oracle against mode 0 at the reference's benchmark
size (473 x 297 points, 3 ghosts, 30 layers) over 10 steps.

Usage (on a machine with a CUDA GPU, after oracle/ref_build.sh):
    python tests/golden/make_meke_golden.py [--out DIR]
"""

from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from more_benchmarks_dc_ocean_b200 import meke_inputs as MI  # noqa: E402
from oracle import meke_oracle as MO  # noqa: E402

REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libmeke_refcuda.so")
HERE = os.path.dirname(os.path.abspath(__file__))
NSTEPS = 3

_PTRS = ("meke", "kh_diff", "le", "ku", "i_mass", "depth_tot", "bottom_fac2", "barotr_fac2", "src", "uflux",
         "vflux", "mass_ws", "rd_ws", "sn_u_ws", "sn_v_ws", "ke_diss_ws", "u_bbl2", "f_centre", "gm_src",
         "ke_diss_ext", "h_layer", "rho_layer", "areaT", "iareaT", "idxT", "idyT", "dy_cu", "dx_cv", "idxCu",
         "idyCv")


class RefArgs(C.Structure):
    """struct MekeArgs as meke/meke_args.h:38-52 lays it out."""

    _fields_ = ([(n, C.c_void_p) for n in _PTRS] + [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int)] +
                [(n, C.c_double) for n in MI.SCALARS[:-1]] + [("backscatter", C.c_int)])


REF_OUTPUTS = tuple(k for k in MI.OUTPUTS if k != "del2")


def cases():
    return [
        ("meke_reference_ic_24x18x6", MI.reference_ic(18, 12, 6)),
        ("meke_all_terms_21x16x11", MI.random_case(21, 16, 11, 201, **MI.all_terms())),
        ("meke_cfl_clip_17x13x9", MI.random_case(17, 13, 9, 202, negative_fraction=0.3, kh_bg=4000.0,
                                                 khmeke_fac=5.0, cdrag=0.0, gmcoeff=-1.0, frcoeff=0.3)),
        ("meke_vanished_16x9x16", MI.random_case(16, 9, 16, 203, land_fraction=0.4, vanished_fraction=0.3,
                                                 min_gamma2=1.5, uscale=0.05, damping=1.0e-5)),
        ("meke_strip_12x2x3", MI.random_case(12, 2, 3, 204, **MI.all_terms())),
        ("meke_closures_off_15x11x8", MI.random_case(15, 11, 8, 205, gmcoeff=-1.0, frcoeff=0.0, khcoeff=0.0,
                                                     backscatter=1, visc_coeff_ku=0.5, bgsrc=2.0e-9)),
    ]


def _ref():
    L = C.CDLL(REF_LIB)
    L.meke_cuda_launch.argtypes = [C.POINTER(RefArgs), C.c_int]
    L.meke_cuda_launch.restype = None
    L.meke_cuda_graph_reset.restype = None
    L.meke_opt_launch.argtypes = [C.POINTER(RefArgs), C.c_void_p]
    L.meke_opt_launch.restype = None
    return L


def _device(p, torch):
    return {k: torch.from_numpy(v).cuda() for k, v in p.arrays.items()}


def _args(p, d):
    a = RefArgs()
    for n in _PTRS:
        setattr(a, n, d[n].data_ptr())
    a.nx, a.ny, a.nz = p.nx, p.ny, p.nz
    for n in MI.SCALARS[:-1]:
        setattr(a, n, float(p.config[n]))
    a.backscatter = int(p.config["backscatter"])
    return a


def run_reference(L, p, nsteps, mode, torch):
    """Outputs after each step of the reference launcher (mode 0/1/2, or 'opt')."""
    d = _device(p, torch)
    a = _args(p, d)
    scratch = torch.zeros(p.ny, p.nx, dtype=torch.float64, device="cuda")
    out = []
    for _ in range(nsteps):
        if mode == "opt":
            L.meke_opt_launch(C.byref(a), scratch.data_ptr())
        else:
            L.meke_cuda_launch(C.byref(a), mode)
        torch.cuda.synchronize()
        out.append({k: d[k].cpu().numpy() for k in REF_OUTPUTS})
    if mode == 2:
        L.meke_cuda_graph_reset()
    return out


def _agree(x, y, keys):
    return all(np.array_equal(a[k], b[k]) for a, b in zip(x, y) for k in keys)


def main():
    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    L = _ref()
    report = {"cases": {}}
    for name, p in cases():
        ref = run_reference(L, p, NSTEPS, 0, torch)
        rec = {"mode1_equals_mode0": _agree(ref, run_reference(L, p, NSTEPS, 1, torch), REF_OUTPUTS),
               "mode2_equals_mode0": _agree(ref, run_reference(L, p, NSTEPS, 2, torch), REF_OUTPUTS),
               "opt_meke_equals_mode0": _agree(ref, run_reference(L, p, NSTEPS, "opt", torch), ("meke",))}
        q = p.copy()
        ok = True
        for s in range(NSTEPS):
            MO.step(q, 1)
            ok = ok and all(np.array_equal(q.arrays[k], ref[s][k]) for k in REF_OUTPUTS)
        rec["oracle_equals_mode0"] = ok
        report["cases"][name] = rec
        z = {"name": np.array(name), "nx": p.nx, "ny": p.ny, "nz": p.nz, "nsteps": NSTEPS}
        z.update({"in_" + k: v for k, v in p.arrays.items()})
        z.update({"cfg_" + k: np.float64(v) for k, v in p.config.items()})
        for s in range(NSTEPS):
            z.update({f"ref_step{s + 1}_{k}": ref[s][k] for k in REF_OUTPUTS})
        np.savez_compressed(os.path.join(args.out, name + ".npz"), **z)
        print(name, rec, flush=True)

    # the oracle against the reference at the benchmark size, 10 steps
    p = MI.reference_ic()
    ref = run_reference(L, p, 10, 0, torch)
    q = p.copy()
    worst = {}
    for s in range(10):
        MO.step(q, 1)
        for k in REF_OUTPUTS:
            d = float(np.abs(q.arrays[k] - ref[s][k]).max())
            worst[k] = max(worst.get(k, 0.0), d)
    report["reference_ic_479x303x30_10_steps"] = {"max_abs_diff": worst,
                                                  "bit_identical": all(v == 0.0 for v in worst.values())}
    print("benchmark size:", report["reference_ic_479x303x30_10_steps"], flush=True)
    with open(os.path.join(args.out, "golden_report_meke.json"), "w") as f:
        json.dump(report, f, indent=1)


if __name__ == "__main__":
    main()
