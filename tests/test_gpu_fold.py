"""The fused Phase-B pass (face flux + fold in one launch) against the CPU oracle, through the C-ABI.

Every tile shape (1 or 2 cell rows) and tracers-per-pass choice (1, 2, 4) must give the
oracle's tracers bit for bit: the fold adds exactly the reference's terms in the
reference's W, E, S, N / ks order. Cases cover the seamount domain, open edges with the
scalar diffusivity, columns of 1 to 7 layers, many tracers (several passes of a launch),
row bands (the host-state step) and tiles cut by the domain edge.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU-only container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from more_benchmarks_dc_ocean_b200 import autotune, inputs  # noqa: E402
from oracle import oracle as O  # noqa: E402


@pytest.fixture
def fold_setting(redi_lib):
    saved = autotune.get_fold()
    yield
    autotune.set_fold(*saved)


def _step_gpu(R, p, nsteps=1, scalar_khtr=False):
    dp = R.to_device(p)
    redi = R.make_redi(dp)
    for _ in range(nsteps):
        assert R.redi_calc_coeffs(dp.grid, dp.metrics, dp.eos, redi, dp.ms) == R.OK
        if scalar_khtr:
            redi.khtr = 1000.0
            assert R.redi_apply_flux(dp.grid, dp.metrics, redi, dp.ms, dp.dt, None, None, dp.bc) == R.OK
        else:
            assert R.redi_apply_flux(dp.grid, dp.metrics, redi, dp.ms, dp.dt, dp.khtr_u_ext, dp.khtr_v_ext,
                                     dp.bc) == R.OK
    torch.cuda.synchronize()
    assert redi.error_count() == 0
    redi.destroy()
    return [t.cpu().numpy() for t in dp.ms.tracers]


def _step_oracle(p, nsteps=1, scalar_khtr=False):
    q = p.copy()
    if scalar_khtr:
        q.khtr_u = np.full_like(q.khtr_u, 1000.0)
        q.khtr_v = np.full_like(q.khtr_v, 1000.0)
    O.step(q, nsteps)
    return q.tracers


def _exact(name, got, ref):
    for n, (a, b) in enumerate(zip(got, ref)):
        if not np.array_equal(a, b):
            pytest.fail(f"{name} tracer {n}: {int(np.count_nonzero(a != b))} values differ, "
                        f"max |diff| {np.abs(a - b).max():.3e}")


@pytest.mark.parametrize("rows,tracers", [(2, 0), (1, 0), (2, 1), (1, 2), (2, 4)])
def test_fold_shapes_match_oracle(redi_lib, oracle_lib, fold_setting, rows, tracers):
    """Config 0 over two steps and a 7-tracer domain whose width is not a multiple of the tile."""
    autotune.set_fold(True, rows, tracers)
    p = inputs.config0()
    _exact(f"config0 rows={rows} nt={tracers}", _step_gpu(redi_lib, p, 2), _step_oracle(p, 2))
    q = inputs.make_problem(47, 23, 9, n_passive=5, seed=31)
    _exact(f"7 tracers rows={rows} nt={tracers}", _step_gpu(redi_lib, q), _step_oracle(q))


@pytest.mark.parametrize("nz", [1, 2, 3, 7])
def test_fold_short_columns(redi_lib, oracle_lib, fold_setting, nz):
    autotune.set_fold(True, 2, 0)
    p = inputs.make_problem(35, 14, nz, n_seamounts=3, seed=70 + nz)
    _exact(f"nz={nz}", _step_gpu(redi_lib, p), _step_oracle(p))


def test_fold_open_edges_scalar_khtr(redi_lib, oracle_lib, fold_setting):
    """No walls on three edges (the tile-edge faces there carry flux) and the scalar khtr path."""
    autotune.set_fold(True, 2, 0)
    p = inputs.make_problem(40, 33, 11, seed=12)
    p.walls = (0, 1, 0, 0)
    _exact("open edges", _step_gpu(redi_lib, p, scalar_khtr=True), _step_oracle(p, scalar_khtr=True))


def test_fold_equals_the_face_flux_gather_pair(redi_lib, fold_setting):
    """The fused pass and the pair it replaces give the same bits on a larger seamount domain."""
    p = inputs.make_problem(190, 130, 30, n_seamounts=12, land_fraction=0.3, n_passive=2, seed=99)
    autotune.set_fold(False, 2, 0)
    pair = _step_gpu(redi_lib, p, 2)
    for rows in (1, 2):
        autotune.set_fold(True, rows, 0)
        _exact(f"fold rows={rows} vs pair", _step_gpu(redi_lib, p, 2), pair)


def test_fold_in_row_bands(redi_lib, oracle_lib, fold_setting):
    """The host-state step runs the fused pass band by band (tile rows clipped at band edges)."""
    R = redi_lib
    autotune.set_fold(True, 2, 0)
    p = inputs.make_problem(41, 37, 8, n_seamounts=4, seed=55)
    ref = _step_oracle(p)
    for nbands in (3, 7):
        dp = R.to_device(p)
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()  # noqa: E731
        host = R.MultilayerState(p.nz, pin(p.h), [pin(t) for t in p.tracers], p.idx_temperature + 1,
                                 p.idx_salinity + 1)
        redi = R.make_redi(dp)
        rc = R.redi_step_host(dp.grid, dp.metrics, dp.eos, redi, host, dp.dt, dp.khtr_u_ext, dp.khtr_v_ext,
                              dp.bc, nbands)
        assert rc == R.OK
        torch.cuda.synchronize()
        assert redi.error_count() == 0
        redi.destroy()
        _exact(f"{nbands} bands", [t.numpy() for t in host.tracers], ref)
