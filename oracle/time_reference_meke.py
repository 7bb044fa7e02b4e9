"""TEST INFRASTRUCTURE ONLY: the reference's own MEKE CUDA against this repository's kernels.

Times the reference's launchers `meke_cuda_launch` modes 0 (faithful, 16
kernels), 1 (fused, 6) and 2 (graph) and `meke_opt_launch` (3 kernels), compiled
from the reference sources with the reference's own flags for sm_100a by
oracle/ref_build.sh into oracle/_ref/libmeke_refcuda_native.so, and this
repository's exports of the same symbols (libredi_b200.so), on identical device
arrays of the reference's benchmark state. Every launcher synchronises the
device before returning; each call is bracketed by CUDA events after a 256 MB
write that evicts the L2, so all of them pay one host round trip and start
cold. The stream-ordered handle call (meke_b200_step) is timed the same way.

    python oracle/time_reference_meke.py [--size 473x297x30] [--reps N]

Prints one JSON line. Needs a GPU and the libraries built.
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

NATIVE = os.path.join(ROOT, "oracle", "_ref", "libmeke_refcuda_native.so")


def main():
    import torch

    from more_benchmarks_dc_ocean_b200 import meke_inputs as MI
    from more_benchmarks_dc_ocean_b200 import ocean_meke as M

    ap = argparse.ArgumentParser()
    ap.add_argument("--size", default="473x297x30", help="points NXxNYxNZ (3 ghost cells are added)")
    ap.add_argument("--reps", type=int, default=50)
    args = ap.parse_args()
    nxp, nyp, nz = (int(v) for v in args.size.split("x"))
    p = MI.reference_ic(nxp, nyp, nz)
    ref = C.CDLL(NATIVE)
    ours = M.lib()
    for L in (ref, ours):
        L.meke_cuda_launch.argtypes = [C.POINTER(M.MekeArgs), C.c_int]
        L.meke_cuda_launch.restype = None
        L.meke_opt_launch.argtypes = [C.POINTER(M.MekeArgs), C.c_void_p]
        L.meke_opt_launch.restype = None
        L.meke_cuda_graph_reset.restype = None
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    clean = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    sink = torch.empty((), dtype=torch.float32, device="cuda")
    out = {"grid_arrays": [p.nx, p.ny, p.nz], "reps": args.reps, "l2": "evicted (write + read) before every call"}

    def timed(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        ts = []
        for i in range(args.reps):
            flush.fill_(float(i))  # evict the L2: a 256 MB write, then a 256 MB read
            torch.sum(clean, dim=0, out=sink)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
        return {"ms_min": round(min(ts), 4), "ms_median": round(float(np.median(ts)), 4)}

    for lib_name, L in (("reference", ref), ("b200", ours)):
        for how in (0, 1, 2, "opt"):
            d = M.to_device(p)
            a = M.make_args(p.nx, p.ny, p.nz, d, p.config)
            scratch = torch.zeros(p.ny, p.nx, dtype=torch.float64, device="cuda")
            if how == "opt":
                r = timed(lambda: L.meke_opt_launch(C.byref(a), scratch.data_ptr()))
            else:
                r = timed(lambda: L.meke_cuda_launch(C.byref(a), how))
            L.meke_cuda_graph_reset()
            out[f"{lib_name}_{'meke_opt_launch' if how == 'opt' else f'meke_cuda_launch_mode{how}'}"] = r
            del d, a, scratch

    d = M.to_device(p)
    h = M.step_problem(p, d, 1)
    a = M.make_args(p.nx, p.ny, p.nz, d, p.config)
    st = torch.cuda.current_stream()
    del2 = C.c_void_p(d["del2"].data_ptr())
    out["b200_meke_b200_step_stream_ordered"] = timed(
        lambda: ours.meke_b200_step(h, C.byref(a), del2, C.c_void_p(st.cuda_stream)))
    M.destroy_handle(h)
    best_ref = min(v["ms_min"] for k, v in out.items() if k.startswith("reference_"))
    out["speedup_b200_opt_vs_reference_best"] = best_ref / out["b200_meke_opt_launch"]["ms_min"]
    out["speedup_b200_stream_vs_reference_best"] = best_ref / out["b200_meke_b200_step_stream_ordered"]["ms_min"]
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
