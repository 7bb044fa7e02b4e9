"""Error of the mixed-precision Redi step against the FP64 step.

    python -m more_benchmarks_dc_ocean_b200.precision_report [--config config1] [--checkpoints 1,100]
                                                            [--control]

Runs the same seeded problem twice on one GPU — the plain FP64 form (which is
bit-identical to the CPU oracle, a restatement of the reference's FP64 code)
and the mixed-precision form — and after each checkpoint step reports, for every
tracer, the max and RMS relative error (|a - b| / max(|a|, |b|), the measure of
redi/drivers/dc_main.F90:228-231), the number of cells above 1e-6, and the max
error relative to the tracer's own change over the run. Prints one JSON line.

--control replaces the mixed-precision run by a second FP64 run whose tracers
start perturbed by a relative 1e-15 (a few ulp, seeded): how far the FP64 step
itself carries a perturbation of that size through its discrete decisions.
"""

from __future__ import annotations

import argparse
import json
import sys

import numpy as np


def compare(a, b) -> dict:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    d = np.abs(a - b)
    sc = np.maximum(np.abs(a), np.abs(b))
    with np.errstate(invalid="ignore", divide="ignore"):
        r = np.where(sc > 1e-30, d / sc, 0.0)
    return {"max_rel": float(r.max()), "rms_rel": float(np.sqrt(np.mean(r * r))),
            "n_above_1e-6": int(np.count_nonzero(r > 1e-6)), "max_abs": float(d.max())}


def run(problem, checkpoints, device="cuda", control=False, eps=1e-15, seed=12345):
    import torch

    from . import ocean_redi as R

    dp64 = R.to_device(problem, device)
    dpm = R.to_device(problem, device)
    r64 = R.make_redi(dp64, R.FP64)
    rm = R.make_redi(dpm, R.FP64 if control else R.MIXED)
    if control:
        g = torch.Generator(device=device).manual_seed(seed)
        for t in dpm.ms.tracers:
            t.mul_(1.0 + eps * (2.0 * torch.rand(t.shape, generator=g, device=device, dtype=t.dtype) - 1.0))
    init = [t.clone() for t in dp64.ms.tracers]
    out = {}
    last = max(checkpoints)
    for step in range(1, last + 1):
        R.step(dp64, r64, 1)
        R.step(dpm, rm, 1)
        if step in checkpoints:
            torch.cuda.synchronize()
            rec = {}
            for n, (a, b, t0) in enumerate(zip(dp64.ms.tracers, dpm.ms.tracers, init)):
                c = compare(a.cpu().numpy(), b.cpu().numpy())
                change = float((a - t0).abs().max().item())
                c["max_abs_over_max_change"] = c["max_abs"] / change if change > 0 else None
                rec[f"tracer{n}"] = c
            out[f"step{step}"] = rec
    r64.destroy()
    rm.destroy()
    return out


def main(argv=None):
    from . import inputs

    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="config1")
    ap.add_argument("--grid", default=None, help="NXxNYxNZ instead of --config")
    ap.add_argument("--checkpoints", default="1,100")
    ap.add_argument("--control", action="store_true", help="FP64 with 1e-15-perturbed tracers instead of mixed")
    args = ap.parse_args(argv)
    if args.grid:
        nx, ny, nz = (int(v) for v in args.grid.split("x"))
        p = inputs.make_problem(nx, ny, nz)
    else:
        p = getattr(inputs, args.config)()
    cps = sorted({int(c) for c in args.checkpoints.split(",")})
    res = run(p, cps, control=args.control)
    second = "fp64 with tracers perturbed by 1e-15 relative" if args.control else "mixed precision"
    print(json.dumps({"workload": p.name, "tracers": p.ntr, "checkpoints": cps, "compared": f"fp64 vs {second}",
                      "errors": res}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
