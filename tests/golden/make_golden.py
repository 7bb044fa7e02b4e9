"""Generate the golden vectors that pin the CPU oracle.

Runs the reference's own CUDA launchers — `redi_opt_launch` (redi/opt_kernel.cu)
and `redi_cuda_launch_` (redi/redi_kernel.cu), built from the reference sources
by oracle/ref_build.sh into oracle/_ref/libredi_refcuda.so with FMA contraction
off — on a GPU, on small seeded inputs, and stores inputs and outputs as
compressed .npz fixtures beside this script. tests/test_oracle_golden.py checks
the CPU oracle against them on any machine.

It also compares the oracle with the reference launchers at the full config-0
size (10 steps) and prints the agreement.

Usage (on a machine with a CUDA GPU, after oracle/ref_build.sh):
    python tests/golden/make_golden.py [--out DIR] [--config0]
"""

from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from more_benchmarks_dc_ocean_b200 import inputs  # noqa: E402
from oracle import oracle as O  # noqa: E402

REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libredi_refcuda.so")
HERE = os.path.dirname(os.path.abspath(__file__))


def cases():
    """Small, fixture-sized problems covering the branches the reference tests and the ones it does not."""
    out = []
    out.append(("seamounts_16x12x6", inputs.make_problem(16, 12, 6, n_seamounts=3, land_fraction=0.15, seed=101)))
    out.append(("reference_ic_20x14x8", inputs.reference_ic(20, 14, 8)))
    out.append(("short_column_10x8x2", inputs.make_problem(10, 8, 2, n_seamounts=2, land_fraction=0.2, seed=7)))
    p = inputs.make_problem(12, 10, 5, n_seamounts=3, land_fraction=0.4, seed=21)
    rng = np.random.default_rng(0)
    mask = rng.random(p.h.shape) < 0.15
    p.h[mask] = 0.0
    for t in p.tracers:
        t[mask] = 0.0
    p.name = "vanished_layers_12x10x5"
    out.append((p.name, p))
    p = inputs.make_problem(14, 10, 7, n_seamounts=2, land_fraction=0.1, seed=33)
    p.walls = (0, 1, 0, 0)
    p.name = "open_edges_14x10x7"
    out.append((p.name, p))
    return out


def _ref_lib():
    if not os.path.exists(REF_LIB):
        raise SystemExit(f"{REF_LIB} missing: run oracle/ref_build.sh where the reference sources are mounted")
    L = C.CDLL(REF_LIB)
    for n in ("redi_opt_launch", "redi_cuda_launch_"):
        getattr(L, n).restype = None
    return L


def run_reference(p, nsteps: int, symbol: str):
    """The reference launcher on torch device memory; returns (coeffs after the last step, tracers per step)."""
    import torch

    L = _ref_lib()
    dev = "cuda"

    def d(a, dtype=torch.float64):
        return torch.from_numpy(np.ascontiguousarray(a)).to(dev, dtype)

    nx, ny, nz, ns = p.nx, p.ny, p.nz, p.ns
    h, T, S = d(p.h), d(p.tracers[0]), d(p.tracers[1])
    wet_u, wet_v = d(p.wet_u), d(p.wet_v)
    c = {}
    for side, (a, b) in (("u", (ny, nx + 1)), ("v", (ny + 1, nx))):
        c[side + "PoL"] = torch.zeros((ns, a, b), dtype=torch.float64, device=dev)
        c[side + "PoR"] = torch.zeros((ns, a, b), dtype=torch.float64, device=dev)
        c[side + "KoL"] = torch.ones((ns, a, b), dtype=torch.int32, device=dev)
        c[side + "KoR"] = torch.ones((ns, a, b), dtype=torch.int32, device=dev)
        c[side + "hEff"] = torch.zeros((ns - 1, a, b), dtype=torch.float64, device=dev)
    ku_ext, kv_ext = d(p.khtr_u), d(p.khtr_v)
    ku, kv = torch.zeros_like(ku_ext), torch.zeros_like(kv_ext)
    metr = [d(p.dy_cu), d(p.dx_cv), d(p.idxCu), d(p.idyCv), d(p.areaT)]
    snap = torch.zeros_like(T)
    ci = lambda v: C.byref(C.c_int(int(v)))  # noqa: E731
    cd = lambda v: C.byref(C.c_double(float(v)))  # noqa: E731
    vp = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    ww, we, ws, wn = p.walls
    e = p.eos
    hist = []
    for _ in range(nsteps):
        getattr(L, symbol)(ci(nx), ci(ny), ci(nz), ci(ns), cd(p.dt), ci(p.nghost), ci(p.nx_phys), ci(p.ny_phys),
                           ci(ww), ci(we), ci(ws), ci(wn), cd(e.rho0), cd(e.T_ref), cd(e.S_ref), cd(e.alpha_T),
                           cd(e.beta_S), vp(h), vp(T), vp(S), vp(wet_u), vp(wet_v),
                           vp(c["uPoL"]), vp(c["uPoR"]), vp(c["uKoL"]), vp(c["uKoR"]), vp(c["uhEff"]),
                           vp(c["vPoL"]), vp(c["vPoR"]), vp(c["vKoL"]), vp(c["vKoR"]), vp(c["vhEff"]),
                           vp(ku_ext), vp(kv_ext), vp(ku), vp(kv), *[vp(m) for m in metr], vp(snap))
        torch.cuda.synchronize()
        hist.append([T.cpu().numpy(), S.cpu().numpy()])
    return {k: v.cpu().numpy() for k, v in c.items()}, hist


def compare(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    d = np.abs(a - b)
    sc = np.maximum(np.abs(a), np.abs(b))
    with np.errstate(invalid="ignore", divide="ignore"):
        r = np.where(sc > 1e-30, d / sc, 0.0)
    return {"equal": bool(np.array_equal(a, b)), "n_diff": int(np.count_nonzero(a != b)),
            "max_abs": float(d.max(initial=0)), "max_rel": float(r.max(initial=0))}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--config0", action="store_true", help="also compare at config 0 (10 steps)")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    report = {}
    for name, p in cases():
        c_opt, h_opt = run_reference(p, args.steps, "redi_opt_launch")
        c_fai, h_fai = run_reference(p, args.steps, "redi_cuda_launch_")
        # the two reference launchers are bit-identical by design (opt_kernel.cu:4-6)
        ident = all(np.array_equal(a, b) for s1, s2 in zip(h_opt, h_fai) for a, b in zip(s1, s2))
        q = p.copy()
        co = O.new_coeffs(p.nx, p.ny, p.nz)
        rec = {"launchers_identical": ident}
        for s in range(args.steps):
            O.calc_coeffs(q, co)
            if s == args.steps - 1:
                for k in co:
                    rec[f"coeff_{k}"] = compare(co[k], c_opt[k])
            O.apply_flux(q, co)
            for n in range(2):
                rec[f"step{s + 1}_tracer{n}"] = compare(q.tracers[n], h_opt[s][n])
        report[name] = rec
        ww, we, ws, wn = p.walls
        np.savez_compressed(
            os.path.join(args.out, f"{name}.npz"),
            nx_phys=p.nx_phys, ny_phys=p.ny_phys, nz=p.nz, nghost=p.nghost, dt=p.dt,
            eos=np.array([p.eos.rho0, p.eos.T_ref, p.eos.S_ref, p.eos.alpha_T, p.eos.beta_S]),
            walls=np.array([ww, we, ws, wn]), h=p.h, T0=p.tracers[0], S0=p.tracers[1],
            dy_cu=p.dy_cu, dx_cv=p.dx_cv, idxCu=p.idxCu, idyCv=p.idyCv, areaT=p.areaT,
            wet_u=p.wet_u, wet_v=p.wet_v, khtr_u=p.khtr_u, khtr_v=p.khtr_v, nsteps=args.steps,
            **{f"ref_{k}": v for k, v in c_opt.items()},
            **{f"ref_step{s + 1}_T": h_opt[s][0] for s in range(args.steps)},
            **{f"ref_step{s + 1}_S": h_opt[s][1] for s in range(args.steps)})
        print(name, json.dumps(rec), flush=True)
    if args.config0:
        p = inputs.config0()
        t0 = time.time()
        _, hist = run_reference(p, 10, "redi_opt_launch")
        t_ref = time.time() - t0
        q = p.copy()
        t0 = time.time()
        O.step(q, 10)
        t_or = time.time() - t0
        rec = {f"step10_tracer{n}": compare(q.tracers[n], hist[-1][n]) for n in range(2)}
        rec["ref_wall_s"], rec["oracle_wall_s"], rec["oracle_threads"] = t_ref, t_or, O.max_threads()
        report["config0_10steps"] = rec
        print("config0_10steps", json.dumps(rec), flush=True)
    with open(os.path.join(args.out, "golden_report.json"), "w") as f:
        json.dump(report, f, indent=1)


if __name__ == "__main__":
    main()
