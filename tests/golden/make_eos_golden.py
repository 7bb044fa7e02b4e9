"""Generate the golden vectors that pin the oracle's Wright (1997) EOS derivatives.

The reference's Redi CUDA evaluates the LINEAR equation of state only, but two
other models of the reference carry a CUDA transcription of eos_specvol_derivs
with the WRIGHT_97 branch (redi/ocean_eos.F90): epbl/epbl_kernel.cu:112-137 and
kappa_shear/ks_kernel.cu:108-134. oracle/ref_build.sh compiles each of them
where it lies, through oracle/ref_eos_harness.cu, with FMA contraction off,
into oracle/_ref/libeos_{epbl,ks}_refcuda.so. This script runs both on seeded
points (T, S, p) over and beyond the oceanic range, for the WRIGHT_97 and the
LINEAR variant, and stores the points and dSV/dT, dSV/dS of each copy in
eos_specvol_ref.npz beside this script (tests/test_oracle_eos.py checks the
oracle against it on any machine; tests/test_gpu_eos.py checks the device EOS).

The reference's ROQUET_SPV derivatives exist in no compiled form of the
reference (the EPBL copy returns zeros for that branch, the kappa-shear copy
has no such branch), so they are not pinned here.

It also records, in golden_report_eos.json, whether the two reference copies
agree with each other and whether the oracle and this repository's
redi_b200_eos_points agree with them.

Usage (on a machine with a CUDA GPU, after oracle/ref_build.sh):
    python tests/golden/make_eos_golden.py [--out DIR]
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

HERE = os.path.dirname(os.path.abspath(__file__))
COPIES = ("epbl", "ks")
VARIANTS = {1: "linear", 2: "wright"}
LINEAR = dict(rho0=1035.0, alpha_T=2.0e-4, beta_S=7.6e-4)


def points(n_random: int = 2048, seed: int = 20260):
    """A 9 x 6 x 5 grid over the oceanic range plus seeded points beyond it."""
    Tg, Sg, pg = np.meshgrid(np.linspace(-2.0, 32.0, 9), np.array([0.0, 5.0, 30.0, 34.7, 35.0, 40.0]),
                             np.array([0.0, 1.0e5, 1.0e7, 4.0e7, 6.0e7]), indexing="ij")
    r = np.random.default_rng(seed)
    T = np.concatenate([Tg.ravel(), r.uniform(-2.5, 40.0, n_random)])
    S = np.concatenate([Sg.ravel(), r.uniform(0.0, 42.0, n_random)])
    p = np.concatenate([pg.ravel(), r.uniform(0.0, 1.1e8, n_random)])
    return T, S, p


def run_reference(copy: str, variant: int, T, S, p):
    lib = C.CDLL(os.path.join(ROOT, "oracle", "_ref", f"libeos_{copy}_refcuda.so"))
    f = lib.ref_eos_specvol_derivs
    dp = C.POINTER(C.c_double)
    f.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, dp, dp, dp, dp, dp]
    f.restype = C.c_int
    n = T.size
    dT, dS = np.empty(n), np.empty(n)
    ptr = lambda a: a.ctypes.data_as(dp)  # noqa: E731
    rc = f(variant, LINEAR["rho0"], LINEAR["alpha_T"], LINEAR["beta_S"], n, ptr(T), ptr(S), ptr(p), ptr(dT), ptr(dS))
    if rc != 0:
        raise RuntimeError(f"ref_eos_specvol_derivs ({copy}, variant {variant}) returned CUDA error {rc}")
    return dT, dS


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    T, S, p = points()
    out = {"T": T, "S": S, "p": p, **{f"cfg_{k}": np.float64(v) for k, v in LINEAR.items()}}
    for v, name in VARIANTS.items():
        for copy in COPIES:
            dT, dS = run_reference(copy, v, T, S, p)
            out[f"{copy}_{name}_dsv_dt"] = dT
            out[f"{copy}_{name}_dsv_ds"] = dS
    np.savez_compressed(os.path.join(args.out, "eos_specvol_ref.npz"), **out)

    report = {"points": int(T.size)}
    for name in VARIANTS.values():
        report[f"{name}_copies_agree"] = all(
            np.array_equal(out[f"epbl_{name}_{d}"], out[f"ks_{name}_{d}"]) for d in ("dsv_dt", "dsv_ds"))

    from more_benchmarks_dc_ocean_b200.inputs import Eos
    from oracle import oracle as O

    for v, name in VARIANTS.items():
        e = Eos(variant=v, **LINEAR)
        got = np.array([O.eos_point(e, a, b, c)[1:] for a, b, c in zip(T, S, p)])
        report[f"{name}_oracle_differs"] = {
            d: int(np.count_nonzero(got[:, i] != out[f"epbl_{name}_{d}"])) for i, d in enumerate(("dsv_dt", "dsv_ds"))}

    import torch

    from more_benchmarks_dc_ocean_b200 import ocean_redi as R

    dev = lambda a: torch.from_numpy(a).cuda()  # noqa: E731
    for v, name in VARIANTS.items():
        _, dT, dS = R.eos_points(R.OceanEos(variant=v, **LINEAR), dev(T), dev(S), dev(p))
        torch.cuda.synchronize()
        report[f"{name}_device_differs"] = {
            d: int(np.count_nonzero(t.cpu().numpy() != out[f"epbl_{name}_{d}"]))
            for d, t in (("dsv_dt", dT), ("dsv_ds", dS))}
    with open(os.path.join(args.out, "golden_report_eos.json"), "w") as f:
        json.dump(report, f, indent=1)
    print(json.dumps(report))


if __name__ == "__main__":
    main()
