"""Uneven regional domains stepped by one persistent kernel, through the C-ABI.

Every domain of a batch must come out exactly as if it had been stepped on its
own: bit-identical to the CPU oracle in FP64, bit-identical to the handle API
at the same precision in both FP64 and mixed form, whatever the launch shape,
with or without the CUDA graph. A domain whose input is never published makes
the step end with a timeout status (bounded waits), and the next step runs.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU-only container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from more_benchmarks_dc_ocean_b200 import inputs  # noqa: E402
from oracle import oracle as O  # noqa: E402

# Odd extents (PPM offsets off any power of two), nz from 1 to 25, 6 tracers.
SHAPES = [(21, 17, 5), (33, 25, 9), (40, 31, 12), (16, 29, 25), (57, 19, 7), (12, 12, 3), (9, 40, 1), (30, 30, 16)]


def _domains():
    ps = [inputs.make_problem(a, b, c, n_seamounts=3, land_fraction=0.2, n_passive=4, seed=900 + d,
                              name=f"d{d}_{a}x{b}x{c}") for d, (a, b, c) in enumerate(SHAPES)]
    ps[3].walls = (0, 1, 0, 0)  # open west / south / north edges on one domain
    return ps


def _assert_exact(name, a, b):
    a, b = np.asarray(a), np.asarray(b)
    if not np.array_equal(a, b):
        d = np.abs(a - b)
        pytest.fail(f"{name}: {int(np.count_nonzero(a != b))} values differ, max |diff| {d.max():.3e}")


def _batch_run(R, ps, nsteps, precision=0, occupancy=0, account=False, **kw):
    dps = [R.to_device(p) for p in ps]
    b = R.RediBatch(dps, precision=precision, **kw)
    if occupancy:
        b.set_tuning(b.tile, b.chunk, occupancy)
        assert b.get_tuning()["occupancy"] == occupancy
    if account:
        b.set_accounting(True)
    b.step(nsteps)
    torch.cuda.synchronize()
    st = b.status()
    if account:  # every tile of the last step is accounted for, once
        tiles = sum(v["tiles"] for v in b.stage_times().values())
        assert tiles == b.items, (tiles, b.items)
    b.destroy()
    assert st["status"] == 0 and st["bad"] == 0, st
    return [[t.cpu().numpy() for t in dp.ms.tracers] for dp in dps]


def _handle_run(R, p, nsteps, precision=0):
    dp = R.to_device(p)
    redi = R.make_redi(dp, precision)
    R.step(dp, redi, nsteps)
    torch.cuda.synchronize()
    assert redi.error_count() == 0
    redi.destroy()
    return [t.cpu().numpy() for t in dp.ms.tracers]


def test_batch_fp64_matches_oracle(redi_lib, oracle_lib):
    """Two steps of eight uneven domains in one launch each: every tracer equals the oracle's, 0 ulp."""
    ps = _domains()
    got = _batch_run(redi_lib, ps, 2)
    for p, g in zip(ps, got):
        q = p.copy()
        O.step(q, 2)
        for n, (a, b) in enumerate(zip(g, q.tracers)):
            _assert_exact(f"{p.name} tracer {n}", a, b)


@pytest.mark.parametrize("tile,chunk,graph,occ", [((32, 4), 8, False, 0), ((16, 8), 4, True, 5),
                                                  ((128, 1), 16, True, 6), ((8, 16), 8, True, 0)])
def test_batch_launch_shapes_identical(redi_lib, tile, chunk, graph, occ):
    """Results do not depend on the gather tile, the vertical chunk, the register budget or the graph."""
    ps = _domains()
    ref = _batch_run(redi_lib, ps, 1)
    got = _batch_run(redi_lib, ps, 1, occupancy=occ, account=True, tile=tile, chunk=chunk, use_graph=graph)
    for p, a, b in zip(ps, got, ref):
        for n in range(len(a)):
            _assert_exact(f"{p.name} tracer {n} tile {tile} chunk {chunk} graph {graph} occ {occ}", a[n], b[n])


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_matches_single_domain_handle(redi_lib, precision):
    """Per domain, the batch equals the handle API at the same precision (FP64 and mixed), bit for bit."""
    ps = _domains()[:5]
    got = _batch_run(redi_lib, ps, 2, precision=precision)
    for p, g in zip(ps, got):
        ref = _handle_run(redi_lib, p, 2, precision)
        for n, (a, b) in enumerate(zip(g, ref)):
            _assert_exact(f"{p.name} tracer {n} precision {precision}", a, b)


def test_batch_mixed_close_to_oracle(redi_lib, oracle_lib):
    """Mixed form after one step: relative error per domain at most 1e-7 of each tracer's scale."""
    ps = _domains()
    got = _batch_run(redi_lib, ps, 1, precision=1)
    for p, g in zip(ps, got):
        q = p.copy()
        O.step(q, 1)
        for n, (a, b) in enumerate(zip(g, q.tracers)):
            scale = max(float(np.abs(b).max()), 1e-300)
            err = float(np.abs(a - b).max()) / scale
            assert err <= 1e-7, f"{p.name} tracer {n}: {err:.3e}"


def test_batch_timeout_is_reported_and_recoverable(redi_lib):
    """A held domain's tiles give up after the wait limit; the status names it; the next step runs clean."""
    R = redi_lib
    ps = _domains()
    dps = [R.to_device(p) for p in ps]
    b = R.RediBatch(dps)
    b.set_wait_limit(20_000_000)  # 20 ms
    b.hold(2)
    b.step()
    st = b.status()
    assert st["status"] == R.STATUS_TIMEOUT, st
    assert st["domain"] == 2 and st["stage"] in (0, 1), st
    b.hold(2, False)
    b.step()
    assert b.status()["status"] == 0
    b.destroy()


def test_batch_rejects_bad_arguments(redi_lib):
    R = redi_lib
    p = inputs.make_problem(12, 10, 4, seed=1)
    dp = R.to_device(p)
    with pytest.raises(R.RediError, match="128 cells"):
        R.RediBatch([dp], tile=(16, 4))
    with pytest.raises(R.RediError, match="chunk"):
        R.RediBatch([dp], chunk=5)
    dp1 = R.to_device(p, tracers=p.tracers[:1])
    dp1.ms.idx_salinity = 0
    with pytest.raises(R.RediError, match="tracers"):
        R.RediBatch([dp1])
    dp.khtr_u_ext = None
    with pytest.raises(R.RediError, match="NULL"):
        R.RediBatch([dp])
