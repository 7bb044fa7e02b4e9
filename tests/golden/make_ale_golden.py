"""Generate the golden vectors that pin the ALE remap CPU oracle.

Runs the reference's own CUDA launcher `ale_remap_cuda` (ale_remap/ale_kernel.cu,
fused = 0: one kernel per production loop), built from the reference sources by
oracle/ref_build.sh into oracle/_ref/libale_refcuda.so with FMA contraction off,
on small seeded cases, and stores inputs and the outputs after every step as
compressed .npz fixtures beside this script (tests/test_ale_cpu.py checks the
oracle against them on any machine, tests/test_gpu_ale.py the sm_100a kernels).

The reference's CUDA remaps T and S with PPM and has no KE rescale, so the
cases are PPM, two tracers, KE rescale off; PCM, PLM, passive tracers and the
rescale are pinned by the oracle restatement alone.

It also records, in golden_report_ale.json, whether the reference's fused form
(fused = 1) and `ale_remap_opt` (ale_remap/opt_kernel.cu) agree with the faithful
form on each case, and the oracle against the faithful form at the reference's
benchmark size (473 x 297 points, 3 ghosts, 30 layers, h-drift 25 %).

Usage (on a machine with a CUDA GPU, after oracle/ref_build.sh):
    python tests/golden/make_ale_golden.py [--out DIR]
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

from more_benchmarks_dc_ocean_b200 import ale_inputs as AI  # noqa: E402
from oracle import ale_oracle as AO  # noqa: E402

REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libale_refcuda.so")
HERE = os.path.dirname(os.path.abspath(__file__))
NSTEPS = 2
OUT = ("h_layer", "tracer0", "tracer1", "u", "v", "mass_budget", "heat_budget", "salt_budget", "bt_eta", "total_h",
       "h_ref", "h_old", "target_h")


def cases():
    return [
        ("ale_reference_ic_26x20x8", AI.reference_ic(20, 14, 8)),
        ("ale_uneven_21x17x12", AI.random_case(21, 17, 12, 401, n_passive=0)),
        ("ale_vanished_16x12x9", AI.random_case(16, 12, 9, 402, n_passive=0, vanished=0.45, zero_targets=3)),
        ("ale_three_layers_12x9x3", AI.random_case(12, 9, 3, 403, n_passive=0, zero_targets=0)),
        ("ale_two_layers_10x8x2", AI.random_case(10, 8, 2, 404, n_passive=0, zero_targets=0)),
        ("ale_one_layer_9x7x1", AI.random_case(9, 7, 1, 405, n_passive=0, zero_targets=0)),
        ("ale_strip_15x1x6", AI.random_case(15, 1, 6, 406, n_passive=0)),
        ("ale_deep_13x11x40", AI.random_case(13, 11, 40, 407, n_passive=0, zero_targets=4)),
    ]


def _ref():
    L = C.CDLL(REF_LIB)
    L.ale_remap_cuda.argtypes = [C.c_int] * 5 + [C.c_void_p] * 15
    L.ale_remap_cuda.restype = None
    L.ale_remap_opt.argtypes = [C.c_int] * 3 + [C.c_void_p] * 13
    L.ale_remap_opt.restype = None
    L.cuda_sync.restype = None
    return L


def run_reference(L, p, nsteps, mode, torch):
    """Outputs after each step of the reference launcher: mode 0 / 1 (ale_remap_cuda fused flag) or 'opt'."""
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    g = {k: d(getattr(p, k)) for k in ("h_layer", "u", "v", "mass_budget", "heat_budget", "salt_budget", "bt_eta",
                                       "bt_H_ref", "dsig", "total_h", "h_ref", "h_old", "target_h")}
    g["tracer0"], g["tracer1"] = d(p.tracers[0]), d(p.tracers[1])
    P = lambda k: g[k].data_ptr()  # noqa: E731
    out = []
    for _ in range(nsteps):
        if mode == "opt":
            L.ale_remap_opt(p.nx, p.ny, p.nz, P("h_layer"), P("h_old"), P("target_h"), P("tracer0"), P("tracer1"),
                            P("u"), P("v"), P("mass_budget"), P("heat_budget"), P("salt_budget"), P("bt_eta"),
                            P("bt_H_ref"), P("dsig"))
        else:
            L.ale_remap_cuda(p.nx, p.ny, p.nz, 3, mode, P("h_layer"), P("h_old"), P("target_h"), P("total_h"),
                             P("h_ref"), P("tracer0"), P("tracer1"), P("u"), P("v"), P("mass_budget"),
                             P("heat_budget"), P("salt_budget"), P("bt_eta"), P("bt_H_ref"), P("dsig"))
        L.cuda_sync()
        torch.cuda.synchronize()
        out.append({k: g[k].cpu().numpy() for k in OUT})
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
    no_ws = tuple(k for k in OUT if k not in ("total_h", "h_ref"))
    for name, p in cases():
        ref = run_reference(L, p, NSTEPS, 0, torch)
        rec = {"fused_equals_faithful": _agree(ref, run_reference(L, p, NSTEPS, 1, torch), OUT),
               "opt_equals_faithful": _agree(ref, run_reference(L, p, NSTEPS, "opt", torch), no_ws)}
        q = p.copy()
        ok = True
        for s in range(NSTEPS):
            AO.step(q, 1)
            got = q.arrays()
            ok = ok and all(np.array_equal(got[k], ref[s][k]) for k in OUT)
        rec["oracle_equals_faithful"] = ok
        report["cases"][name] = rec
        z = {"name": np.array(name), "nx": p.nx, "ny": p.ny, "nz": p.nz, "nsteps": NSTEPS}
        for k in ("h_layer", "u", "v", "mass_budget", "heat_budget", "salt_budget", "bt_eta", "bt_H_ref", "dsig"):
            z["in_" + k] = getattr(p, k)
        z["in_tracer0"], z["in_tracer1"] = p.tracers
        for s in range(NSTEPS):
            z.update({f"ref_step{s + 1}_{k}": ref[s][k] for k in OUT})
        np.savez_compressed(os.path.join(args.out, name + ".npz"), **z)
        print(name, rec, flush=True)

    p = AI.reference_ic()
    ref = run_reference(L, p, 1, 0, torch)
    q = p.copy()
    AO.step(q, 1)
    got = q.arrays()
    worst = {k: float(np.abs(got[k] - ref[0][k]).max()) for k in OUT}
    report["reference_ic_479x303x30_drift25"] = {"max_abs_diff": worst,
                                                 "bit_identical": all(v == 0.0 for v in worst.values())}
    print("benchmark size:", report["reference_ic_479x303x30_drift25"], flush=True)
    with open(os.path.join(args.out, "golden_report_ale.json"), "w") as f:
        json.dump(report, f, indent=1)


if __name__ == "__main__":
    main()
