"""GPU parity: the sm_100a FP64 path against the CPU oracle, through the C-ABI.

The plain FP64 form is compiled with FMA contraction off and keeps the
reference's operation order, so the bar is exact equality (0 ulp) on every
coefficient and every tracer value, after one and after several steps. The
reference's own tolerance for cross-implementation agreement is 1e-12 relative
(redi/drivers/dc_main.F90:228-237); a failure message reports that figure too.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU-only container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from more_benchmarks_dc_ocean_b200 import inputs  # noqa: E402
from oracle import oracle as O  # noqa: E402

REL_BAR = 1e-12


def _rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    sc = np.maximum(np.abs(a), np.abs(b))
    d = np.abs(a - b)
    with np.errstate(invalid="ignore", divide="ignore"):
        r = np.where(sc > 1e-30, d / sc, 0.0)
    return float(d.max(initial=0.0)), float(r.max(initial=0.0))


def _assert_exact(name, gpu, ref):
    gpu = np.asarray(gpu)
    ref = np.asarray(ref)
    assert gpu.shape == ref.shape, (name, gpu.shape, ref.shape)
    if not np.array_equal(gpu, ref):
        dmax, rmax = _rel(gpu, ref)
        nbad = int(np.count_nonzero(gpu != ref))
        pytest.fail(f"{name}: {nbad} values differ; max|diff| {dmax:.3e} max rel {rmax:.3e} (bar 0 ulp, ref bar {REL_BAR})")


def _run_gpu(p, nsteps, redi_lib, check_coeffs=True):
    R = redi_lib
    dp = R.to_device(p)
    redi = R.make_redi(dp)
    for _ in range(nsteps):
        assert R.redi_calc_coeffs(dp.grid, dp.metrics, dp.eos, redi, dp.ms) == R.OK
        assert R.redi_apply_flux(dp.grid, dp.metrics, redi, dp.ms, dp.dt, dp.khtr_u_ext, dp.khtr_v_ext, dp.bc) == R.OK
    torch.cuda.synchronize()
    coeffs = {k: v.cpu().numpy() for k, v in redi.coeffs().items()} if check_coeffs else None
    trs = [t.cpu().numpy() for t in dp.ms.tracers]
    assert redi.error_count() == 0
    redi.destroy()
    return coeffs, trs


def _run_oracle(p, nsteps):
    q = p.copy()
    c = O.step(q, nsteps)
    return c, q.tracers


def _compare(p, nsteps, redi_lib):
    cg, tg = _run_gpu(p, nsteps, redi_lib)
    co, to = _run_oracle(p, nsteps)
    for k in ("uPoL", "uPoR", "uKoL", "uKoR", "uhEff", "vPoL", "vPoR", "vKoL", "vKoR", "vhEff"):
        _assert_exact(f"{p.name} {k}", cg[k], co[k])
    for n, (a, b) in enumerate(zip(tg, to)):
        _assert_exact(f"{p.name} tracer {n} after {nsteps} steps", a, b)


def test_config0_one_step(redi_lib, oracle_lib):
    _compare(inputs.config0(), 1, redi_lib)


def test_config0_ten_steps(redi_lib, oracle_lib):
    """Config 0 (128x96x25): 10 steps compared against the FP64 oracle."""
    _compare(inputs.config0(), 10, redi_lib)


def test_reference_ic_small(redi_lib, oracle_lib):
    """The reference driver's own IC (dc_main.F90:172-206) at a reduced size."""
    _compare(inputs.reference_ic(40, 30, 12), 3, redi_lib)


@pytest.mark.parametrize("nz", [1, 2, 3, 4, 7])
def test_short_columns(redi_lib, oracle_lib, nz):
    """PCM ends, the nk<=2 edge cases of redi_interface_scalar and the sweep."""
    _compare(inputs.make_problem(17, 13, nz, n_seamounts=3, land_fraction=0.2, seed=11 + nz), 2, redi_lib)


def test_open_boundaries_and_scalar_khtr(redi_lib, oracle_lib):
    """Non-WALL edges (flux crosses into the halo) and the scalar-khtr path (no ext arrays)."""
    p = inputs.make_problem(24, 20, 9, seed=5)
    p.walls = (0, 1, 0, 0)
    R = redi_lib
    dp = R.to_device(p)
    redi = R.make_redi(dp)
    redi.khtr = 1000.0
    for _ in range(2):
        R.redi_calc_coeffs(dp.grid, dp.metrics, dp.eos, redi, dp.ms)
        R.redi_apply_flux(dp.grid, dp.metrics, redi, dp.ms, dp.dt, None, None, dp.bc)
    torch.cuda.synchronize()
    tg = [t.cpu().numpy() for t in dp.ms.tracers]
    redi.destroy()
    co, to = _run_oracle(p, 2)  # khtr_u/v arrays hold 1000 everywhere: same per-face values
    for n, (a, b) in enumerate(zip(tg, to)):
        _assert_exact(f"open/scalar tracer {n}", a, b)


def test_uniform_fields_tie_break(redi_lib, oracle_lib):
    """Horizontally uniform T/S: dRho == 0 everywhere, the sweep's tie-break branch."""
    p = inputs.make_problem(12, 10, 6, n_seamounts=0, land_fraction=0.0, seed=3)
    p.h[:] = 100.0
    zc = (np.arange(6)[::-1] + 0.5) * 100.0
    for n, base in enumerate((10.0, 35.0)):
        p.tracers[n][:] = (base + 0.001 * zc)[:, None, None] * 100.0
    _compare(p, 2, redi_lib)


def test_vanished_layers_and_land(redi_lib, oracle_lib):
    """Zero-thickness layers (PCM next to vanished layers, H_DIV_EPS floors) and large land fraction."""
    p = inputs.make_problem(20, 16, 8, n_seamounts=4, land_fraction=0.5, seed=21)
    rng = np.random.default_rng(0)
    mask = rng.random(p.h.shape) < 0.15
    p.h[mask] = 0.0
    for t in p.tracers:
        t[mask] = 0.0
    _compare(p, 2, redi_lib)


def test_many_tracers_fused(redi_lib, oracle_lib):
    """T, S and passive tracers in one fused apply (odd count exercises partial groups)."""
    _compare(inputs.make_problem(30, 22, 10, n_passive=5, seed=9), 2, redi_lib)


def test_compat_launcher_matches_oracle(redi_lib, oracle_lib):
    """redi_opt_launch / redi_cuda_launch_ exports, called like the reference bridge."""
    R = redi_lib
    for symbol in ("redi_opt_launch", "redi_cuda_launch_"):
        p = inputs.make_problem(26, 18, 11, seed=13)
        dp = R.to_device(p)
        nx, ny, nz, ns = p.nx, p.ny, p.nz, p.ns
        c = {}
        for side, (a, b) in (("u", (ny, nx + 1)), ("v", (ny + 1, nx))):
            c[side + "PoL"] = torch.zeros((ns, a, b), dtype=torch.float64, device="cuda")
            c[side + "PoR"] = torch.zeros((ns, a, b), dtype=torch.float64, device="cuda")
            c[side + "KoL"] = torch.ones((ns, a, b), dtype=torch.int32, device="cuda")
            c[side + "KoR"] = torch.ones((ns, a, b), dtype=torch.int32, device="cuda")
            c[side + "hEff"] = torch.zeros((ns - 1, a, b), dtype=torch.float64, device="cuda")
        ku = torch.zeros_like(dp.khtr_u_ext)
        kv = torch.zeros_like(dp.khtr_v_ext)
        snap = torch.zeros_like(dp.ms.tracers[0])
        m = dp.metrics
        R.redi_opt_launch(nx, ny, nz, p.dt, p.nghost, p.nx_phys, p.ny_phys, (1, 1, 1, 1), dp.eos, dp.ms.h_layer,
                          dp.ms.tracers[0], dp.ms.tracers[1], m.wet_u, m.wet_v, c, dp.khtr_u_ext, dp.khtr_v_ext,
                          ku, kv, m.dy_cu, m.dx_cv, m.idxCu, m.idyCv, m.areaT, snap, symbol=symbol)
        co, to = _run_oracle(p, 1)
        for k in co:
            _assert_exact(f"{symbol} {k}", c[k].cpu().numpy(), co[k])
        for n in range(2):
            _assert_exact(f"{symbol} tracer {n}", dp.ms.tracers[n].cpu().numpy(), to[n])
        assert torch.equal(ku, dp.khtr_u_ext) and torch.equal(kv, dp.khtr_v_ext)


def test_gates_are_noops(redi_lib):
    """The reference's early returns: disabled handle, unregistered T/S, nz mismatch, khtr<=0 without ext."""
    R = redi_lib
    p = inputs.make_problem(10, 8, 5, seed=2)
    dp = R.to_device(p)
    before = [t.clone() for t in dp.ms.tracers]
    redi = R.OceanRedi()
    redi.init(dp.grid, p.nz)
    assert R.redi_calc_coeffs(dp.grid, dp.metrics, dp.eos, redi, dp.ms) == R.SKIPPED  # enable = .false.
    redi.enable = True
    ms2 = R.MultilayerState(p.nz, dp.ms.h_layer, dp.ms.tracers, 0, 2)
    assert R.redi_calc_coeffs(dp.grid, dp.metrics, dp.eos, redi, ms2) == R.SKIPPED
    ms3 = R.MultilayerState(p.nz + 1, dp.ms.h_layer, dp.ms.tracers, 1, 2)
    assert R.redi_calc_coeffs(dp.grid, dp.metrics, dp.eos, redi, ms3) == R.SKIPPED
    assert R.redi_apply_flux(dp.grid, dp.metrics, redi, dp.ms, p.dt, None, None, None) == R.SKIPPED  # khtr = 0
    torch.cuda.synchronize()
    for a, b in zip(before, dp.ms.tracers):
        assert torch.equal(a, b)
    redi.destroy()


def test_invalid_arguments_raise(redi_lib):
    R = redi_lib
    p = inputs.make_problem(10, 8, 5, seed=2)
    dp = R.to_device(p)
    redi = R.make_redi(dp)
    bad = R.HGrid(p.nx + 1, p.ny, p.nx_phys, p.ny_phys, p.nghost)
    with pytest.raises(R.RediError):
        R.redi_calc_coeffs(bad, dp.metrics, dp.eos, redi, dp.ms)
    eos = R.OceanEos(variant=3)  # EOS_VARIANT_TEOS10: reserved in the reference (ocean_eos.F90:49)
    with pytest.raises(R.RediError):
        R.redi_calc_coeffs(dp.grid, dp.metrics, eos, redi, dp.ms)
    redi.destroy()
    with pytest.raises(R.RediError):
        R.OceanRedi().init(dp.grid, 4096)


@pytest.mark.parametrize("tile,chunk", [((32, 4), 4), ((64, 2), 8), ((128, 1), 16), ((32, 1), 8)])
def test_cell_update_launch_shapes_are_bit_identical(redi_lib, oracle_lib, tile, chunk):
    """Every tile shape and vertical chunk of the cell update gives the reference's result."""
    from more_benchmarks_dc_ocean_b200 import autotune

    saved = autotune.get_tuning()
    try:
        autotune.set_tuning(tile[0], tile[1], chunk)
        _compare(inputs.make_problem(37, 29, 23, n_passive=1, seed=31), 2, redi_lib)
    finally:
        autotune.set_tuning(*saved)


def test_autotuner_picks_a_candidate(redi_lib, tmp_path, monkeypatch):
    from more_benchmarks_dc_ocean_b200 import autotune

    monkeypatch.setenv("REDI_B200_TUNING_CACHE", str(tmp_path / "t.json"))
    saved = autotune.get_tuning()
    try:
        p = inputs.make_problem(40, 30, 12, seed=4)
        R = redi_lib
        dp = R.to_device(p)
        redi = R.make_redi(dp)
        res = autotune.tune(dp, redi, candidates=[(32, 4, 8), (64, 2, 4)], reps=1)
        assert res["best"] in [(32, 4, 8), (64, 2, 4)] and not res["cached"]
        assert autotune.get_tuning() == res["best"]
        again = autotune.tune(dp, redi, candidates=[(32, 4, 8), (64, 2, 4)], reps=1)
        assert again["cached"] and again["best"] == res["best"]
        redi.destroy()
    finally:
        autotune.set_tuning(*saved)


def test_mixed_precision_first_step_close_to_fp64(redi_lib, oracle_lib):
    """Mixed form: every decision input is the FP64 one, so one step differs from the
    oracle only by FP32 rounding of the layer means and the flux: relative error
    ~1e-7 of a cell's own change, well under the 1e-6 bar on the tracer."""
    from more_benchmarks_dc_ocean_b200 import precision_report as PR

    R = redi_lib
    p = inputs.config0()
    dp = R.to_device(p)
    redi = R.make_redi(dp, R.MIXED)
    R.step(dp, redi, 1)
    torch.cuda.synchronize()
    got = [t.cpu().numpy() for t in dp.ms.tracers]
    assert redi.error_count() == 0
    redi.destroy()
    _, ref = _run_oracle(p, 1)
    for n in range(2):
        c = PR.compare(got[n], ref[n])
        assert c["max_rel"] <= 1e-7, (n, c)
        assert c["n_above_1e-6"] == 0


def test_mixed_precision_many_tracers_and_gates(redi_lib, oracle_lib):
    """Mixed form with passive tracers (several tracer groups) and the scalar-khtr path."""
    from more_benchmarks_dc_ocean_b200 import precision_report as PR

    R = redi_lib
    p = inputs.make_problem(30, 22, 10, n_passive=9, seed=19)
    dp = R.to_device(p)
    redi = R.make_redi(dp, R.MIXED)
    redi.khtr = 1000.0
    R.redi_calc_coeffs(dp.grid, dp.metrics, dp.eos, redi, dp.ms)
    R.redi_apply_flux(dp.grid, dp.metrics, redi, dp.ms, dp.dt, None, None, dp.bc)
    torch.cuda.synchronize()
    got = [t.cpu().numpy() for t in dp.ms.tracers]
    with pytest.raises(R.RediError):
        redi.coeffs()  # packed mixed-precision slots are not exposed in the reference layout
    redi.destroy()
    _, ref = _run_oracle(p, 1)
    for n in range(len(ref)):
        # passive tracers cross zero, so compare against each field's scale
        scale = np.abs(ref[n]).max()
        assert np.abs(got[n] - ref[n]).max() <= 1e-7 * scale, n


@pytest.mark.parametrize("gnt,smem,chunk", [(2, 1, 4), (2, 1, 8), (2, 1, 16), (4, 0, 4), (4, 1, 8), (2, 2, 8),
                                            (2, 2, 16), (4, 2, 4), (8, 1, 4), (8, 2, 4), (8, 1, 8), (2, 3, 4),
                                            (2, 3, 8), (2, 3, 16), (4, 3, 4), (4, 3, 8)])
def test_gather_forms_match_oracle(redi_lib, oracle_lib, gnt, smem, chunk):
    """The gather folding 2, 4 or 8 tracers per launch (8: two face-flux launches of 4 into one
    flux buffer; with 8-layer chunks it falls back to 4), with its per-layer sums in registers or
    in shared memory: the same additions in the same order, so the oracle's bits."""
    from more_benchmarks_dc_ocean_b200 import autotune

    saved = (autotune.get_tuning(), autotune.get_gather_tracers(), autotune.get_tracer_group())
    try:
        autotune.set_tuning(64, 2, chunk)
        autotune.set_gather_tracers(gnt, smem)
        autotune.set_tracer_group(4)
        p = inputs.make_problem(45, 27, 19, n_passive=5 if gnt < 8 else 8, seed=23)
        _, tg = _run_gpu(p, 1, redi_lib, check_coeffs=False)
        _, to = _run_oracle(p, 1)
        for n, (a, b) in enumerate(zip(tg, to)):
            _assert_exact(f"gather gnt={gnt} smem={smem} chunk={chunk} tracer {n}", a, b)
    finally:
        autotune.set_tuning(*saved[0])
        autotune.set_gather_tracers(*saved[1])
        autotune.set_tracer_group(saved[2])


@pytest.mark.parametrize("form,group,precision", [(1, 1, 0), (1, 2, 0), (1, 2, 1), (2, 1, 0), (2, 2, 0), (2, 4, 0),
                                                   (2, 2, 1), (2, 4, 1)])
def test_staged_face_flux_matches(redi_lib, oracle_lib, form, group, precision):
    """The face flux with its reconstruction staged through shared memory one sublayer ahead
    (form 1) or read through a two-layer ring per column side (form 2): FP64 equals the oracle
    bit for bit; the mixed form equals the plain mixed form bit for bit."""
    from more_benchmarks_dc_ocean_b200 import autotune

    R = redi_lib
    saved = (autotune.get_flux_staged(), autotune.get_tracer_group())
    p = inputs.make_problem(43, 29, 17, n_passive=3, seed=61)
    try:
        autotune.set_tracer_group(group)
        if precision:
            autotune.set_flux_staged(False)
            dp = R.to_device(p)
            redi = R.make_redi(dp, R.MIXED)
            R.step(dp, redi, 1)
            torch.cuda.synchronize()
            ref = [t.cpu().numpy() for t in dp.ms.tracers]
            redi.destroy()
            autotune.set_flux_staged(form)
            dp = R.to_device(p)
            redi = R.make_redi(dp, R.MIXED)
            R.step(dp, redi, 1)
            torch.cuda.synchronize()
            got = [t.cpu().numpy() for t in dp.ms.tracers]
            assert redi.error_count() == 0
            redi.destroy()
        else:
            autotune.set_flux_staged(form)
            _, got = _run_gpu(p, 1, redi_lib, check_coeffs=False)
            _, ref = _run_oracle(p, 1)
        for n, (a, b) in enumerate(zip(got, ref)):
            _assert_exact(f"flux form={form} group={group} precision={precision} tracer {n}", a, b)
    finally:
        autotune.set_flux_staged(saved[0])
        autotune.set_tracer_group(saved[1])


_SWEEP_CASES = {
    "config0": lambda: inputs.config0(),
    "tie_break": lambda: _uniform_problem(),
    "vanished": lambda: _vanished_problem(),
    "nz1": lambda: inputs.make_problem(17, 13, 1, n_seamounts=3, land_fraction=0.2, seed=12),
    "nz2": lambda: inputs.make_problem(17, 13, 2, n_seamounts=3, land_fraction=0.2, seed=13),
}


def _uniform_problem():
    p = inputs.make_problem(12, 10, 6, n_seamounts=0, land_fraction=0.0, seed=3)
    p.h[:] = 100.0
    zc = (np.arange(6)[::-1] + 0.5) * 100.0
    for n, base in enumerate((10.0, 35.0)):
        p.tracers[n][:] = (base + 0.001 * zc)[:, None, None] * 100.0
    return p


def _vanished_problem():
    p = inputs.make_problem(20, 16, 8, n_seamounts=4, land_fraction=0.5, seed=21)
    mask = np.random.default_rng(0).random(p.h.shape) < 0.15
    p.h[mask] = 0.0
    for t in p.tracers:
        t[mask] = 0.0
    return p


@pytest.mark.parametrize("form", [0, 3, 4, 5])
@pytest.mark.parametrize("case", sorted(_SWEEP_CASES))
def test_sweep_forms_match_oracle(redi_lib, oracle_lib, form, case):
    """Every neutral-sweep form (register windows; windows in a shared-memory ring of 3, 4 or 5
    interfaces) gives the oracle's coefficients and tracers bit for bit over two steps."""
    from more_benchmarks_dc_ocean_b200 import autotune

    saved = autotune.get_sweep_form()
    try:
        autotune.set_sweep_form(form)
        _compare(_SWEEP_CASES[case](), 2, redi_lib)
    finally:
        autotune.set_sweep_form(saved)


@pytest.mark.parametrize("form", [3, 4, 5])
def test_sweep_forms_mixed_match_register_form(redi_lib, form):
    """The mixed-precision step (FP64 sweep decisions, narrower coefficient storage) does not
    depend on the sweep form either: tracers after two steps equal bit for bit."""
    from more_benchmarks_dc_ocean_b200 import autotune

    R = redi_lib
    saved = autotune.get_sweep_form()
    p = inputs.make_problem(41, 33, 23, n_seamounts=5, land_fraction=0.3, seed=77)
    out = []
    try:
        for f in (0, form):
            autotune.set_sweep_form(f)
            dp = R.to_device(p)
            redi = R.make_redi(dp, R.MIXED)
            R.step(dp, redi, 2)
            torch.cuda.synchronize()
            assert redi.error_count() == 0
            out.append([t.cpu().numpy() for t in dp.ms.tracers])
            redi.destroy()
    finally:
        autotune.set_sweep_form(saved)
    for n, (a, b) in enumerate(zip(out[1], out[0])):
        _assert_exact(f"mixed sweep form {form} tracer {n}", a, b)


def test_sweep_form_rejects_unknown(redi_lib):
    from more_benchmarks_dc_ocean_b200 import autotune

    with pytest.raises(Exception):
        autotune.set_sweep_form(2)


@pytest.mark.parametrize("case", ["tie_break", "vanished", "nz1", "nz2"])
def test_ring_face_flux_edge_cases(redi_lib, oracle_lib, case):
    """The ring face flux on the sweep's edge cases (uniform fields, vanished layers and land,
    one- and two-layer columns), two steps, bit for bit."""
    from more_benchmarks_dc_ocean_b200 import autotune

    saved = autotune.get_flux_staged()
    try:
        autotune.set_flux_staged(2)
        _compare(_SWEEP_CASES[case](), 2, redi_lib)
    finally:
        autotune.set_flux_staged(saved)


def test_dry_faces_follow_changing_masks(redi_lib, oracle_lib):
    """Faces that turn dry or wet between steps, and slots overwritten by the caller: the handle's
    record of dry faces (faces whose slots hold inert coefficients are not rewritten, and are not
    walked by Phase B) follows the masks, and handing out the slots clears it. Coefficients and
    tracers equal the oracle's after every step."""
    R = redi_lib
    p = inputs.make_problem(31, 23, 9, n_seamounts=3, land_fraction=0.3, seed=91)
    q = p.copy()
    q.wet_u, q.wet_v = p.wet_u.copy(), p.wet_v.copy()
    dp = R.to_device(p)
    redi = R.make_redi(dp)
    rng = np.random.default_rng(5)
    c = None
    for step in range(4):
        if step in (1, 2):  # flip a tenth of the faces both ways
            fu = rng.random(q.wet_u.shape) < 0.1
            fv = rng.random(q.wet_v.shape) < 0.1
            q.wet_u[fu] = 1.0 - q.wet_u[fu]
            q.wet_v[fv] = 1.0 - q.wet_v[fv]
            dp.metrics.wet_u.copy_(torch.from_numpy(q.wet_u))
            dp.metrics.wet_v.copy_(torch.from_numpy(q.wet_v))
        if step == 3:  # the caller writes into the slots it was handed (the oracle's too: the
            # domain-edge faces, which no sweep writes, keep what the caller put there)
            for k, t in redi.coeffs().items():
                t.fill_(7)
                if k in c:
                    c[k][...] = 7
        assert R.redi_calc_coeffs(dp.grid, dp.metrics, dp.eos, redi, dp.ms) == R.OK
        assert R.redi_apply_flux(dp.grid, dp.metrics, redi, dp.ms, dp.dt, dp.khtr_u_ext, dp.khtr_v_ext,
                                 dp.bc) == R.OK
        torch.cuda.synchronize()
        c = O.step(q, 1, coeffs=c)
        cg = {k: v.cpu().numpy() for k, v in redi.coeffs().items()}
        for k in ("uPoL", "uPoR", "uKoL", "uKoR", "uhEff", "vPoL", "vPoR", "vKoL", "vKoR", "vhEff"):
            _assert_exact(f"step {step} {k}", cg[k], c[k])
        for n, (a, b) in enumerate(zip(dp.ms.tracers, q.tracers)):
            _assert_exact(f"step {step} tracer {n}", a.cpu().numpy(), b)
    assert redi.error_count() == 0
    redi.destroy()


def test_apply_flux_before_any_coefficients(redi_lib, oracle_lib):
    """redi_apply_flux on a fresh handle: every slot holds the inert coefficients of init, so every
    flux is zero and the tracers come out as the reference's update leaves them."""
    R = redi_lib
    p = inputs.make_problem(19, 15, 6, n_seamounts=2, land_fraction=0.2, seed=17)
    q = p.copy()
    dp = R.to_device(p)
    redi = R.make_redi(dp)
    assert R.redi_apply_flux(dp.grid, dp.metrics, redi, dp.ms, dp.dt, dp.khtr_u_ext, dp.khtr_v_ext, dp.bc) == R.OK
    torch.cuda.synchronize()
    O.apply_flux(q, O.new_coeffs(q.nx, q.ny, q.nz), None, 0)
    for n, (a, b) in enumerate(zip(dp.ms.tracers, q.tracers)):
        _assert_exact(f"fresh handle tracer {n}", a.cpu().numpy(), b)
    redi.destroy()


@pytest.mark.parametrize("case", ["config0", "vanished", "nz1", "nz2", "tie_break", "swapped_ts", "many_tracers"])
@pytest.mark.parametrize("precision", [0, 1])
def test_whole_step_call_matches_two_calls(redi_lib, oracle_lib, case, precision):
    """redi_b200_step (one call; Phase A's column state and the T/S reconstruction in one pass)
    equals redi_calc_coeffs + redi_apply_flux bit for bit over two steps, FP64 and mixed, and the
    FP64 form equals the oracle."""
    R = redi_lib
    if case == "swapped_ts":
        p = inputs.make_problem(29, 21, 11, n_seamounts=3, land_fraction=0.3, seed=44)
        p.tracers = [p.tracers[1], p.tracers[0]]
        p.idx_temperature, p.idx_salinity = p.idx_salinity, p.idx_temperature
    elif case == "many_tracers":
        p = inputs.make_problem(31, 19, 13, n_passive=5, land_fraction=0.3, seed=45)
    else:
        p = _SWEEP_CASES[case]()
    out = []
    for combined in (False, True):
        dp = R.to_device(p)
        redi = R.make_redi(dp, R.MIXED if precision else R.FP64)
        for _ in range(2):
            if combined:
                assert R.redi_step(dp.grid, dp.metrics, dp.eos, redi, dp.ms, dp.dt, dp.khtr_u_ext, dp.khtr_v_ext,
                                   dp.bc) == R.OK
            else:
                assert R.redi_calc_coeffs(dp.grid, dp.metrics, dp.eos, redi, dp.ms) == R.OK
                assert R.redi_apply_flux(dp.grid, dp.metrics, redi, dp.ms, dp.dt, dp.khtr_u_ext, dp.khtr_v_ext,
                                         dp.bc) == R.OK
        torch.cuda.synchronize()
        assert redi.error_count() == 0
        out.append([t.cpu().numpy() for t in dp.ms.tracers])
        redi.destroy()
    for n, (a, b) in enumerate(zip(out[1], out[0])):
        _assert_exact(f"{case} whole-step call tracer {n}", a, b)
    if not precision:
        _, to = _run_oracle(p, 2)
        for n, (a, b) in enumerate(zip(out[1], to)):
            _assert_exact(f"{case} whole-step call vs oracle tracer {n}", a, b)


def test_whole_step_call_gates(redi_lib):
    """redi_b200_step keeps each phase's gates: a disabled handle is SKIPPED."""
    R = redi_lib
    p = inputs.make_problem(12, 10, 5, seed=2)
    dp = R.to_device(p)
    redi = R.make_redi(dp)
    redi.enable = False
    assert R.redi_step(dp.grid, dp.metrics, dp.eos, redi, dp.ms, dp.dt, dp.khtr_u_ext, dp.khtr_v_ext,
                       dp.bc) == R.SKIPPED
    redi.destroy()
