"""Domain decomposition on CPU ranks (gloo): tiles that exchange the one-column
halo of h and every tracer before each step reproduce, on every physical cell,
the undivided domain's result bit for bit (the oracle computes both)."""

import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, nsteps, q):
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from more_benchmarks_dc_ocean_b200 import halo, inputs
    from oracle import oracle as O

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        g = inputs.make_problem(24, 16, 6, n_seamounts=3, land_fraction=0.2, n_passive=1, seed=77)
        t = halo.Tiling.for_world(world, rank)
        tile = halo.global_split(g, t)
        fields = [torch.from_numpy(tile.h)] + [torch.from_numpy(x) for x in tile.tracers]
        ex = halo.HaloExchange(t, fields=fields, nghost=tile.nghost)
        c = O.new_coeffs(tile.nx, tile.ny, tile.nz)
        for _ in range(nsteps):
            ex.exchange()
            O.calc_coeffs(tile, c, nthreads=1)
            O.apply_flux(tile, c, nthreads=1)
        gg = tile.nghost
        q.put((rank, t.tx, t.ty, [x[:, gg:-gg, gg:-gg].copy() for x in tile.tracers]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
def test_tiles_match_undivided_domain(world, oracle_lib):
    from more_benchmarks_dc_ocean_b200 import halo, inputs

    nsteps = 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, nsteps, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    g = inputs.make_problem(24, 16, 6, n_seamounts=3, land_fraction=0.2, n_passive=1, seed=77)
    oracle_lib.step(g, nsteps)
    px, py = halo.factor_tiles(world)
    nxp, nyp = g.nx_phys // px, g.ny_phys // py
    gg = g.nghost
    for rank, tx, ty, trs in got:
        for n, tr in enumerate(trs):
            ref = g.tracers[n][:, gg + ty * nyp: gg + (ty + 1) * nyp, gg + tx * nxp: gg + (tx + 1) * nxp]
            assert np.array_equal(tr, ref), f"rank {rank} tracer {n}"


def test_tiling_geometry():
    from more_benchmarks_dc_ocean_b200 import halo

    assert halo.factor_tiles(8) == (4, 2) and halo.factor_tiles(2) == (2, 1) and halo.factor_tiles(1) == (1, 1)
    t = halo.Tiling.for_world(8, 5)
    assert (t.tx, t.ty) == (1, 1)
    assert t.neighbour(-1, 0) == 4 and t.neighbour(0, -1) == 1 and t.neighbour(0, 1) is None
    assert t.walls() == (0, 0, 0, 1)
