"""The host-state step (redi_b200_step_host) against the device entry points.

A model whose state lives in host memory hands h and its tracers to one call
that streams rows up, steps row bands as soon as their rows are on the device,
and streams finished rows back. Every band reads pre-step tracers and writes a
separate copy, so the result must equal redi_calc_coeffs + redi_apply_flux on
device arrays bit for bit, for any number of bands, in both precisions.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU-only container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from more_benchmarks_dc_ocean_b200 import inputs  # noqa: E402


def _problem(seed=77, open_edge=False):
    p = inputs.make_problem(37, 29, 23, n_seamounts=4, land_fraction=0.2, n_passive=3, seed=seed)
    if open_edge:
        p.walls = (1, 0, 1, 0)
    return p


def _device_result(R, p, nsteps, precision):
    dp = R.to_device(p)
    redi = R.make_redi(dp, precision)
    R.step(dp, redi, nsteps)
    torch.cuda.synchronize()
    coeffs = {k: v.cpu().numpy() for k, v in redi.coeffs().items()} if precision == R.FP64 else None
    trs = [t.cpu().numpy() for t in dp.ms.tracers]
    redi.destroy()
    return trs, coeffs


def _host_result(R, p, nsteps, precision, nbands, pinned=True):
    dp = R.to_device(p)  # metrics, masks and diffusivities stay on the device
    hold = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory() if pinned else torch.from_numpy(  # noqa: E731
        np.ascontiguousarray(a).copy())
    ms_host = R.MultilayerState(p.nz, hold(p.h), [hold(t) for t in p.tracers], p.idx_temperature + 1,
                                p.idx_salinity + 1)
    redi = R.make_redi(dp, precision)
    for _ in range(nsteps):
        rc = R.redi_step_host(dp.grid, dp.metrics, dp.eos, redi, ms_host, dp.dt, dp.khtr_u_ext, dp.khtr_v_ext,
                              dp.bc, nbands)
        assert rc == R.OK
    torch.cuda.synchronize()
    coeffs = {k: v.cpu().numpy() for k, v in redi.coeffs().items()} if precision == R.FP64 else None
    assert redi.error_count() == 0
    redi.destroy()
    return [t.numpy().copy() for t in ms_host.tracers], coeffs


@pytest.mark.parametrize("nbands", [1, 3, 8, 29])
def test_host_step_equals_device_step(redi_lib, nbands):
    R = redi_lib
    p = _problem(open_edge=nbands == 3)
    want, cw = _device_result(R, p, 2, R.FP64)
    got, cg = _host_result(R, p, 2, R.FP64, nbands)
    for n, (a, b) in enumerate(zip(got, want)):
        assert np.array_equal(a, b), f"{nbands} bands: tracer {n}"
    for k in cw:
        assert np.array_equal(cg[k], cw[k]), f"{nbands} bands: {k}"


def test_host_step_mixed_precision(redi_lib):
    R = redi_lib
    p = _problem(seed=78)
    want, _ = _device_result(R, p, 2, R.MIXED)
    got, _ = _host_result(R, p, 2, R.MIXED, 5)
    for n, (a, b) in enumerate(zip(got, want)):
        assert np.array_equal(a, b), f"tracer {n}"


def test_host_step_from_pageable_memory(redi_lib):
    R = redi_lib
    p = _problem(seed=79)
    want, _ = _device_result(R, p, 1, R.FP64)
    got, _ = _host_result(R, p, 1, R.FP64, 4, pinned=False)
    for n, (a, b) in enumerate(zip(got, want)):
        assert np.array_equal(a, b), f"tracer {n}"


def test_host_step_gates(redi_lib):
    """A disabled handle skips the call and leaves the host state untouched."""
    R = redi_lib
    p = _problem(seed=80)
    dp = R.to_device(p)
    ms_host = R.MultilayerState(p.nz, torch.from_numpy(p.h.copy()), [torch.from_numpy(t.copy()) for t in p.tracers],
                                p.idx_temperature + 1, p.idx_salinity + 1)
    redi = R.make_redi(dp)
    redi.enable = False
    before = [t.clone() for t in ms_host.tracers]
    assert R.redi_step_host(dp.grid, dp.metrics, dp.eos, redi, ms_host, dp.dt, dp.khtr_u_ext, dp.khtr_v_ext,
                            dp.bc, 4) == R.SKIPPED
    torch.cuda.synchronize()
    assert all(torch.equal(a, b) for a, b in zip(ms_host.tracers, before))
    redi.destroy()
