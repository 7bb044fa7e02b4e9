"""CPU oracle: invariants of the reference algorithm and determinism of the inputs."""

import numpy as np
import pytest

from more_benchmarks_dc_ocean_b200 import inputs


def test_generator_is_deterministic():
    a, b = inputs.config0(), inputs.config0()
    assert np.array_equal(a.h, b.h)
    for x, y in zip(a.tracers, b.tracers):
        assert np.array_equal(x, y)
    assert np.array_equal(a.wet_u, b.wet_u) and np.array_equal(a.wet_v, b.wet_v)


def test_generator_shapes_and_distributions():
    p = inputs.config0()
    assert (p.nx, p.ny, p.nz) == (132, 100, 25)
    assert abs(p.meta["land_fraction"] - 0.15) < 0.02
    assert p.h.min() >= 1e-3
    T = p.tracers[0] / p.h
    S = p.tracers[1] / p.h
    assert 0.0 < T.min() and T.max() < 27.0
    assert 34.0 < S.min() and S.max() < 36.0
    q = inputs.make_problem(360, 270, 10, n_seamounts=40, land_fraction=0.30, n_passive=2, seed=4)
    assert abs(q.meta["land_fraction"] - 0.30) < 0.03
    assert len(q.tracers) == 4
    shapes = inputs.config4_shapes()
    assert len(shapes) == 64
    assert all(64 <= a <= 512 and 64 <= b <= 512 and c in (25, 50, 75) for a, b, c in shapes)


def test_reference_ic_matches_driver_formula():
    p = inputs.reference_ic(20, 14, 8)
    assert p.nghost == 3 and p.dt == 900.0 and p.eos.alpha_T == 1.7e-4
    hh = 4000.0 / 8
    # dc_main.F90:193-202 at ii = jj = 1 (fx = fy = 0), kk = nz (the surface layer)
    zz = 0.5 * hh
    assert p.tracers[0][-1, 0, 0] == (2.0 + 16.0 * np.exp(-zz / 800.0)) * hh


def test_oracle_conserves_tracer_content(oracle_lib):
    p = inputs.make_problem(40, 30, 12, n_passive=1, seed=2)
    before = [t.sum() for t in p.tracers]
    oracle_lib.step(p, 3)
    for b, t in zip(before, p.tracers):
        assert abs(t.sum() - b) <= 1e-12 * abs(b)


def test_oracle_coefficient_invariants(oracle_lib):
    p = inputs.make_problem(30, 24, 9, n_seamounts=4, land_fraction=0.25, seed=8)
    c = oracle_lib.calc_coeffs(p)
    for side, wet in (("u", p.wet_u), ("v", p.wet_v)):
        Ko = np.stack([c[side + "KoL"], c[side + "KoR"]])
        Po = np.stack([c[side + "PoL"], c[side + "PoR"]])
        assert Ko.min() >= 1 and Ko.max() <= p.nz
        assert Po.min() >= 0.0 and Po.max() <= 1.0
        assert c[side + "hEff"].min() >= 0.0
        dry = wet == 0.0
        assert np.all(c[side + "hEff"][:, dry] == 0.0) and np.all(Ko[:, :, dry] == 1)
        # the sweep's positions Ko + Po never move up a column (monotonic backstop, ocean_redi.F90:385-388)
        pos = Ko + Po
        assert np.all(np.diff(pos, axis=1) >= 0.0)
        assert np.all(np.diff(Ko, axis=1) >= 0)
    # faces the reference never visits keep the init values
    assert np.all(c["uKoL"][:, :, 0] == 1) and np.all(c["uKoL"][:, :, -1] == 1)
    assert np.all(c["vKoL"][:, 0, :] == 1) and np.all(c["vKoL"][:, -1, :] == 1)


def test_oracle_thread_count_invariant(oracle_lib):
    p = inputs.make_problem(24, 18, 7, seed=12)
    a, b = p.copy(), p.copy()
    oracle_lib.step(a, 2, nthreads=1)
    oracle_lib.step(b, 2, nthreads=0)
    for x, y in zip(a.tracers, b.tracers):
        assert np.array_equal(x, y)


def test_oracle_op_counts(oracle_lib):
    p = inputs.make_problem(16, 12, 6, seed=3)
    a, b = oracle_lib.count_ops(p)
    assert a["div"] > 0 and b["div"] > 0 and b["add"] > a["add"]
    a2, b2 = oracle_lib.count_ops(p)
    assert a == a2 and b == b2
