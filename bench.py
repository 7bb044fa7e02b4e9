"""Benchmark of the Redi neutral-diffusion step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--config config1|config3|config0|config4] [--precision fp64|mixed]

One step = redi_calc_coeffs + redi_apply_flux over every tracer of the domain (one redi_b200_step
call: the same two phases, with the column state and the T/S reconstruction in one pass).
Metric (the reference's headline): tracer-cell updates/s = N_tracers * nx_phys * ny_phys * nz
/ t_step, land cells included; `value` sums all ranks.

* value: inputs resident in HBM, K steps timed with CUDA events on the
  launching stream between a barrier + synchronize on both sides, max over ranks.
  Every field (0.94 GB per tracer at 1440x1080x75) exceeds the 126 MB L2, so
  no flush is needed between steps.
* e2e: the same metric through the public entry points with the model state
  resident in pinned HOST memory: every step copies h and every tracer host to
  device, runs the step and copies every tracer back. On one GPU this is
  redi_b200_step_host, which pipelines the copies and the kernels over row
  bands; with halo exchange (N > 1) the copies wrap the device entry points.
  On one GPU the line also carries copy_floor_ms, the same copies alone (up
  and down concurrently, no kernels), and e2e's fraction of it.
* roofline: the dominant kernel (most device time in the timed region, from
  CUDA event pairs the library records around each launch on its stream);
  achieved = algorithmic bytes per launch / mean launch time.
* cpu_baseline: the CPU oracle (a restatement of the reference's
  do-concurrent CPU path, OpenMP over all host cores) on a row band of the
  same workload, rank 0 at N=1.
* --impl reference: the reference arm — the same CPU implementation on the
  same workload, timed per step on a bounded row band (the reference's Fortran
  DATA=none build cannot be compiled without a Fortran compiler).

For N > 1 each rank owns one 1440x1080x75 tile of an N-tile global domain
(weak scaling); tiles exchange a halo of h and every tracer with their
neighbours over NCCL before each step (the only data exchange the path has).
"""

from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Redi tracer-cell updates/s, HBM GB/s; mixed+batched vs FP64 plain, 1 B200"
UNIT = "tracer-cell updates/s"
KERNEL_NAMES = ["k_column_state", "k_neutral_sweep", "k_tracer_recon", "k_cell_gather", "k_face_flux",
                "k_mixed_recon", "k_mixed_flux", "k_mixed_sweep", "k_domain_persistent", "aux",
                "k_meke_column", "k_meke_del2", "k_meke_lateral", "k_ale_columns", "k_ale_faces",
                "k_flux_fold", "k_mixed_fold", "k_column_recon"]
NKERN = len(KERNEL_NAMES)
FALLBACK_HBM_GBS = 6650.0


def _rank_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(
        os.environ.get("LOCAL_RANK", "0"))


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def _problem(name: str, grid: str | None = None):
    from more_benchmarks_dc_ocean_b200 import inputs

    if grid:
        nxp, nyp, nz = (int(v) for v in grid.lower().split("x"))
        return inputs.make_problem(nxp, nyp, nz, n_seamounts=40 if nxp * nyp > 200000 else 6,
                                   land_fraction=0.30 if nxp * nyp > 200000 else 0.15, name=f"grid_{grid}")
    return getattr(inputs, name)()


def _sizes(p):
    nx, ny, nz = p.nx, p.ny, p.nz
    return dict(Nt=nx * ny * nz, ncol=nx * ny, Fu=(nx + 1) * ny, Fv=nx * (ny + 1), ns=2 * nz + 2, ntr=p.ntr)


def boundary_bytes(p, precision: str = "fp64") -> float:
    """Algorithmic HBM bytes of one step, boundary model: Phase A reads h, T, S and
    writes the coefficients, Phase B reads h and the coefficients once and
    reads + writes every tracer; plus the 2-D face/cell metrics."""
    s = _sizes(p)
    per_surf = 32 if precision == "fp64" else 24  # Po x2 f64, Ko x2 i32|i16, hEff f64|f32 (ns-1 ~ ns)
    bcoef = (s["Fu"] + s["Fv"]) * s["ns"] * per_surf
    b2d = 8 * (s["Fu"] + s["Fv"]) * 4 + 8 * s["ncol"]
    return 8 * s["Nt"] * (3 + 1 + 2 * s["ntr"]) + 2 * bcoef + b2d


def kernel_bytes(p, kid: int, precision: str = "fp64") -> float:
    """Algorithmic bytes one launch of kernel `kid` must move (its share of the boundary model)."""
    s = _sizes(p)
    per_surf = 32 if precision == "fp64" else 24
    bcoef = (s["Fu"] + s["Fv"]) * s["ns"] * per_surf
    face2d = 8 * (s["Fu"] + s["Fv"]) * 4 + 8 * s["ncol"]
    if kid == 0:   # column state: read h, T, S
        return 24.0 * s["Nt"]
    if kid in (1, 7):  # neutral sweep: write the coefficients
        return float(bcoef)
    if kid in (2, 5):  # tracer reconstruction: read h and every tracer
        return 8.0 * s["Nt"] * (1 + s["ntr"])
    if kid in (4, 6):  # face flux: read the coefficients once for every tracer
        return float(bcoef + face2d)
    if kid == 3:       # cell gather, one launch per tracer pair: read + write its tracers
        return float(16 * s["Nt"] * min(2, s["ntr"]) + 8 * s["ncol"])
    if kid in (15, 16):  # fused face flux + fold: the coefficients once, every tracer read + written
        return float(bcoef + face2d + 16 * s["Nt"] * s["ntr"])
    if kid == 17:        # column state + T/S reconstruction in one pass: read h, T, S once
        return 24.0 * s["Nt"]
    return 0.0


class ClockSampler:
    """Clocks and throttle reasons of one GPU during a timed region: nvidia-smi every 200 ms, and an
    NVML poller every 2 ms for regions shorter than nvidia-smi's period (read-only queries)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # nvmlClocksEventReason* bits
    NVML_BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.proc = None
        self.path = None
        self.nvml = []
        self._stop = None
        self._thread = None

    def _poll_nvml(self):
        try:
            import pynvml as N

            N.nvmlInit()
            h = N.nvmlDeviceGetHandleByUUID(self.uuid) if self.uuid else N.nvmlDeviceGetHandleByIndex(0)
            mx = N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM)
            while not self._stop.is_set():
                sm = N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM)
                rs = N.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.nvml.append((sm, mx, rs))
                self._stop.wait(0.002)
            N.nvmlShutdown()
        except Exception:
            pass

    def start(self):
        import threading

        self._stop = threading.Event()
        self._thread = threading.Thread(target=self._poll_nvml, daemon=True)
        self._thread.start()
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
            if self.uuid:
                cmd.insert(1, f"--id={self.uuid}")
            self.proc = subprocess.Popen(cmd, stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def _nvml_summary(self) -> dict:
        sm = [x[0] for x in self.nvml]
        reasons = sorted({n for x in self.nvml for n, b in self.NVML_BITS.items() if x[2] & b})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(x[1] for x in self.nvml), "reasons": reasons,
                "samples": len(sm), "source": "nvml, 2 ms"}

    def stop(self) -> dict:
        if self._stop is not None:
            self._stop.set()
            self._thread.join(timeout=2)
        rows = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            with open(self.path) as f:
                for line in f:
                    parts = [x.strip() for x in line.split(",")]
                    if len(parts) >= 9:
                        rows.append(parts)
            os.unlink(self.path)
        if not rows:
            if self.nvml:
                return self._nvml_summary()
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        pw = [float(r[3]) for r in rows if re.match(r"^[\d.]+$", r[3])]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        out = {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
               "power_w_max": max(pw) if pw else None, "reasons": reasons, "samples": len(rows)}
        if self.nvml:
            out["nvml"] = self._nvml_summary()
        return out


def _ncu_traffic() -> dict:
    """Per-launch DRAM traffic (bytes) of each kernel at 1440x1080x75, from the committed ncu summaries."""
    out = {}
    d = os.path.join(ROOT, "profiles")
    if not os.path.isdir(d):
        return out
    for fn in os.listdir(d):
        if not fn.endswith(".md"):
            continue
        for line in open(os.path.join(d, fn)):
            m = re.match(r"^traffic_bytes_per_launch_full:\s*(\w+)\s*=\s*([\d.eE+]+)", line.strip())
            if m:
                out[m.group(1)] = float(m.group(2))
    return out


# ---------------------------------------------------------------------------
# CPU oracle sample (cpu_baseline and the reference arm)
# ---------------------------------------------------------------------------
def _row_band(p, nrows: int):
    """Rows [0, nrows) of the physical domain (with its ghost rows) as a standalone problem."""
    from more_benchmarks_dc_ocean_b200.inputs import RediProblem

    g = p.nghost
    ny = nrows + 2 * g
    sl = slice(0, ny)
    return RediProblem(
        name=f"{p.name}_rows{nrows}", nx_phys=p.nx_phys, ny_phys=nrows, nz=p.nz, nghost=g, dt=p.dt, eos=p.eos,
        h=np.ascontiguousarray(p.h[:, sl, :]), tracers=[np.ascontiguousarray(t[:, sl, :]) for t in p.tracers],
        idx_temperature=p.idx_temperature, idx_salinity=p.idx_salinity,
        dy_cu=np.ascontiguousarray(p.dy_cu[sl]), dx_cv=np.ascontiguousarray(p.dx_cv[: ny + 1]),
        idxCu=np.ascontiguousarray(p.idxCu[sl]), idyCv=np.ascontiguousarray(p.idyCv[: ny + 1]),
        areaT=np.ascontiguousarray(p.areaT[sl]), wet_u=np.ascontiguousarray(p.wet_u[sl]),
        wet_v=np.concatenate([p.wet_v[:ny], np.zeros((1, p.nx))]),
        khtr_u=np.ascontiguousarray(p.khtr_u[sl]), khtr_v=np.ascontiguousarray(p.khtr_v[: ny + 1]),
        walls=p.walls, meta=dict(p.meta))


def cpu_sample(p, target_s: float, nsteps: int = 1, warmup: int = 0):
    """Time the oracle on a row band of p sized for ~target_s per step; returns (updates/s, info)."""
    from oracle import oracle as O

    threads = len(os.sched_getaffinity(0))
    probe = _row_band(p, 2)
    t0 = time.perf_counter()
    O.step(probe.copy(), 1, nthreads=threads)
    t_probe = max(time.perf_counter() - t0, 1e-3)
    rows = int(max(1, min(p.ny_phys, math.floor(2 * target_s / t_probe))))
    band = _row_band(p, rows)
    times = []
    for s in range(warmup + nsteps):
        q = band.copy()
        t0 = time.perf_counter()
        O.step(q, 1, nthreads=threads)
        dt = time.perf_counter() - t0
        if s >= warmup:
            times.append(dt)
    t = min(times)
    upd = band.ntr * band.nx_phys * band.ny_phys * band.nz / t
    return upd, {"cores": threads, "rows": rows, "t_step_s": t, "times_s": times,
                 "sample": f"{band.nx_phys}x{rows}x{band.nz} row band of {p.name} ({band.ntr} tracers), "
                           f"min of {len(times)} step(s)"}


# ---------------------------------------------------------------------------
# Reference arm
# ---------------------------------------------------------------------------
def run_reference(args, rank, world):
    if rank != 0:
        return 0
    if args.config == "config4":  # the largest domain of the batch stands for the whole set
        from more_benchmarks_dc_ocean_b200 import inputs

        shapes = inputs.config4_shapes()
        d = max(range(len(shapes)), key=lambda i: shapes[i][0] * shapes[i][1] * shapes[i][2])
        p = inputs.config4_domain(20261203, d, shapes[d])
    else:
        p = _problem(args.config, args.grid)
    budget = 150.0
    per_step = max(2.0, budget / max(1, args.steps + args.warmup))
    upd, info = cpu_sample(p, per_step, nsteps=args.steps, warmup=args.warmup)
    line = {
        "impl": "reference", "metric": METRIC, "value": upd, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": info["t_step_s"] * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": _config_block(p, args, world),
        "cpu_baseline": {"value": upd, "unit": UNIT, "cores": info["cores"], "kind": "port",
                         "sample": info["sample"]},
        "e2e": {"value": upd, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference CPU path (do-concurrent DATA=none restated in C++, OpenMP over all host cores); "
                "the Fortran build itself needs a Fortran compiler, absent on this image",
    }
    print(json.dumps(line), flush=True)
    return 0


def _config_block(p, args, world):
    return {
        "workload": f"{args.grid or args.config}: {'plain FP64' if args.precision == 'fp64' else 'mixed-precision'} Redi step "
                    f"{p.nx_phys}x{p.ny_phys}x{p.nz}, nghost {p.nghost}, {p.ntr} tracers"
                    + (f", {world} tiles" if world > 1 else ""),
        "grid": [p.nx_phys, p.ny_phys, p.nz], "tracers": p.ntr, "dt_s": p.dt, "khtr_m2s": float(p.khtr_u.flat[0]),
        "land_fraction": round(p.meta.get("land_fraction", 0.0), 4), "precision": args.precision,
        "l2": ("inputs larger than L2 (126 MB), no flush" if 8 * p.nx * p.ny * p.nz > 126e6
               else "fields smaller than L2: not a headline configuration"),
        "parallelism": f"dp{world}" if world > 1 else "1 GPU",
    }


# ---------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------
def run_b200(args, rank, world, local_rank):
    import ctypes as C

    import torch

    from more_benchmarks_dc_ocean_b200 import ocean_redi as R

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist  # noqa: F811
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)
    from more_benchmarks_dc_ocean_b200 import halo

    p = _problem(args.config, args.grid)
    tiling = halo.Tiling.for_world(world, rank, p) if world > 1 else None
    if tiling is not None:
        p = tiling.local_problem(p)
    prec = R.FP64 if args.precision == "fp64" else R.MIXED
    if args.fold or args.flux_staged or args.sweep_form is not None:
        from more_benchmarks_dc_ocean_b200 import autotune

        if args.fold:
            autotune.set_fold(autotune.FOLD_FP64 | autotune.FOLD_MIXED)
        if args.flux_staged:
            autotune.set_flux_staged(args.flux_staged)
        if args.sweep_form is not None:
            autotune.set_sweep_form(args.sweep_form)
    dp = R.to_device(p, dev)
    redi = R.make_redi(dp, prec)
    ex = None
    if tiling is not None:
        ex = halo.HaloExchange(tiling, dp)
        ex.setup_masks(dp, p.wet)
        ex.exchange()
    st = torch.cuda.current_stream()
    tuning = None
    if not args.no_tune:
        from more_benchmarks_dc_ocean_b200 import autotune

        tuning = autotune.tune(dp, redi, use_cache=False, stream=st)
        if p.ntr > 2:
            tuning["tracer_group"] = autotune.tune_tracer_group(dp, redi, stream=st)
        if dist is not None:  # every rank uses rank 0's choice
            best = tuple(tuning["best"]) + (0,) * (4 - len(tuning["best"]))
            t = torch.tensor(list(best) + [autotune.get_tracer_group(), autotune.get_gather_tracers()[0]],
                             dtype=torch.int64, device=dev)
            dist.broadcast(t, 0)
            v = [int(x) for x in t.tolist()]
            autotune.set_tuning(*v[:3])
            autotune.set_tracer_group(v[4])
            autotune.set_gather_tracers(v[5], v[3])
            tuning["best"] = tuple(v[:4])
    L = R.lib()
    L.redi_b200_launch_count.restype = C.c_ulonglong
    L.redi_b200_launch_count.argtypes = [C.c_int]

    def one_step():
        if ex is not None:
            ex.exchange()
        R.step(dp, redi, 1, st)

    def barrier():
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        one_step()
    torch.cuda.synchronize()

    # ---- timed region: device-resident inputs ----
    clocks = ClockSampler(_uuid(local_rank))
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    L.redi_b200_profile_begin()
    n0 = L.redi_b200_launch_count(-1)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(args.steps):
        one_step()
    e1.record(st)
    torch.cuda.synchronize()
    n1 = L.redi_b200_launch_count(-1)
    ktime = (C.c_double * NKERN)()
    kcount = (C.c_ulonglong * NKERN)()
    L.redi_b200_profile_end(ktime, kcount, NKERN)
    barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / args.steps
    ms_all = _max_over_ranks(ms, dist, dev)

    upd_per_rank = p.ntr * p.nx_phys * p.ny_phys * p.nz
    value = upd_per_rank * world / (ms_all * 1e-3)
    kern = {KERNEL_NAMES[k]: {"ms_total": ktime[k], "launches": int(kcount[k]),
                              "ms_per_launch": ktime[k] / kcount[k]} for k in range(NKERN) if kcount[k]}
    top = max((k for k in range(NKERN) if kcount[k]), key=lambda k: ktime[k])
    peak, peak_kind = _peaks()
    bytes_launch = kernel_bytes(p, top, args.precision)
    t_launch = ktime[top] / kcount[top] * 1e-3
    achieved = bytes_launch / t_launch / 1e9
    traffic = _ncu_traffic().get(KERNEL_NAMES[top]) if (p.nx_phys, p.ny_phys, p.nz) == (1440, 1080, 75) else None
    bstep = boundary_bytes(p, args.precision)

    # ---- e2e: host-resident state through the public entry points ----
    e2e = None
    if not args.no_e2e:
        e2e = _e2e(args, p, dp, redi, ex, st, dist, dev, world)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        upd, info = cpu_sample(p, args.cpu_seconds / 3, nsteps=3)
        cpu = {"value": upd, "unit": UNIT, "cores": info["cores"], "kind": "port",
               "cores_note": "the threads of this process's CPU affinity set (the lease's cores), one per thread",
               "sample": info["sample"]}

    # ---- the second half of the metric: mixed precision (config 2) and 34-tracer batching (config 3) ----
    sub = None
    if world == 1 and not args.no_sub and args.config == "config1" and args.precision == "fp64" and not args.grid:
        redi.destroy()
        sub = _mixed_batched(args, p, dp, st, value)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_all, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f64+f32", "data": "synthetic",
            "config": _config_block(p, args, world),
            "roofline": {"bound": "hbm", "kernel": KERNEL_NAMES[top], "achieved": achieved, "peak": peak,
                         "peak_source": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "algorithmic_bytes_per_launch": bytes_launch},
            "step_roofline": {"boundary_bytes_per_step": bstep, "achieved_gbs": bstep / (ms_all * 1e-3) / 1e9,
                              "frac": bstep / (ms_all * 1e-3) / 1e9 / peak},
            "kernels": kern,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "clocks": clk,
            "gpu_launches": int(n1 - n0),
            "tuning": {"cell_update_tile": list(tuning["best"][:2]), "vertical_chunk": tuning["best"][2],
                       "gather_sums": {0: "registers", 1: "shared memory", 2: "shared memory, 8-deep batches",
                                       3: "shared memory, pipelined batches of 4"}[
                           tuning["best"][3] if len(tuning["best"]) > 3 else 0],
                       "tracer_group": tuning.get("tracer_group"),
                       "candidates_ms": tuning["ms"]} if tuning else None,
            "hbm_gbs_per_rank": bstep / (ms_all * 1e-3) / 1e9,
        }
        if sub is not None:
            line.update(sub)
        print(json.dumps(line), flush=True)
    redi.destroy()
    if ex is not None:
        ex.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def _time_steps(dp, redi, st, warmup: int, steps: int) -> float:
    """ms per Redi step (calc_coeffs + apply_flux of every tracer), CUDA events on the launching stream."""
    import torch

    from more_benchmarks_dc_ocean_b200 import ocean_redi as R

    for _ in range(warmup):
        R.step(dp, redi, 1, st)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(steps):
        R.step(dp, redi, 1, st)
    e1.record(st)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def _mixed_batched(args, p, dp, st, plain_value: float) -> dict:
    """Sub-records for the mixed+batched half of the metric, measured in this process right after the
    plain line: config 2 (the same 1440x1080x75 inputs, mixed precision) and config 3 (720x576x50, T, S
    and 32 passive tracers, mixed precision, every tracer's fluxes in one fused Phase-B launch). Each
    reports ms per step, tracer-cell updates/s and its ratio to the plain FP64 value of this line."""
    import torch

    from more_benchmarks_dc_ocean_b200 import inputs
    from more_benchmarks_dc_ocean_b200 import ocean_redi as R

    from more_benchmarks_dc_ocean_b200 import autotune

    out = {}
    steps, warm = max(3, min(args.steps, 10)), 3
    saved = (autotune.get_tuning(), autotune.get_gather_tracers())
    redi = R.make_redi(dp, R.MIXED)
    # The FP64 line's gather shape is not the mixed one's best (FP32 fluxes halve the gather's
    # loads), so the mixed step picks its own among the shapes that win in either precision.
    shape2 = autotune.tune(dp, redi, candidates=[(64, 2, 4, 1), (64, 2, 8, 1), (32, 4, 8, 1), (32, 4, 16, 2),
                                                   (64, 2, 16, 2), (64, 2, 16, 3), (32, 4, 8, 3)], reps=1,
                           use_cache=False, stream=st)
    ms = _time_steps(dp, redi, st, warm, steps)
    redi.destroy()
    upd = p.ntr * p.nx_phys * p.ny_phys * p.nz / (ms * 1e-3)
    out["mixed_c2"] = {"workload": f"config2: mixed-precision Redi step {p.nx_phys}x{p.ny_phys}x{p.nz}, "
                                   f"{p.ntr} tracers (the inputs of this line)",
                       "ms_per_step": ms, "value": upd, "unit": UNIT, "steps": steps, "warmup": warm,
                       "ratio_vs_plain": upd / plain_value, "gather_shape": list(shape2["best"]),
                       "gather_shape_ms": shape2["ms"]}
    q = inputs.config3()
    dq = R.to_device(q, torch.device("cuda", torch.cuda.current_device()))
    redi = R.make_redi(dq, R.MIXED)
    shape = autotune.tune(dq, redi, candidates=[(64, 2, 4, 0), (64, 2, 4, 1), (32, 4, 4, 1), (64, 2, 8, 1),
                                                  (32, 4, 8, 1), (32, 4, 4, 2), (32, 4, 8, 2), (32, 4, 8, 3),
                                                  (64, 2, 8, 3), (32, 4, 4, 3)], reps=1,
                          use_cache=False, stream=st)
    group = autotune.tune_tracer_group(dq, redi, stream=st)
    ms = _time_steps(dq, redi, st, warm, steps)
    redi.destroy()
    upd = q.ntr * q.nx_phys * q.ny_phys * q.nz / (ms * 1e-3)
    out["batched_c3"] = {"workload": f"config3: mixed-precision Redi step {q.nx_phys}x{q.ny_phys}x{q.nz}, "
                                     f"{q.ntr} tracers; coefficients once per step, every tracer reconstructed in "
                                     f"one launch, face fluxes in tracer groups of {group['best'][0]}, gathers of "
                                     f"{group['best'][1]} tracers (autotuned)",
                         "ms_per_step": ms, "value": upd, "unit": UNIT, "steps": steps, "warmup": warm,
                         "ratio_vs_plain": upd / plain_value, "tracer_group_ms": group["ms"],
                         "gather_shape": list(shape["best"]), "gather_shape_ms": shape["ms"]}
    autotune.set_tracer_group(8)
    autotune.set_tuning(*saved[0])
    autotune.set_gather_tracers(saved[1][0], saved[1][1])
    del dq
    torch.cuda.empty_cache()
    return out


# ---------------------------------------------------------------------------
# Uneven-domain batch (config4): one persistent kernel over a tile-work queue
# ---------------------------------------------------------------------------
def _domains_config_block(ps, args, world, prec_name):
    shapes = [(p.nx_phys, p.ny_phys, p.nz) for p in ps]
    return {
        "workload": f"config4: {len(ps)} uneven regional domains (nx, ny log-uniform in [64, 512], nz in "
                    f"{{25, 50, 75}}), {ps[0].ntr} tracers each, {prec_name} Redi step, one persistent kernel "
                    "replayed from a CUDA graph" + (f", {world} ranks x {len(ps)} domains" if world > 1 else ""),
        "domains": len(ps), "tracers": ps[0].ntr, "cells": int(sum(a * b * c for a, b, c in shapes)),
        "nx_range": [min(a for a, _, _ in shapes), max(a for a, _, _ in shapes)],
        "ny_range": [min(b for _, b, _ in shapes), max(b for _, b, _ in shapes)],
        "nz_set": sorted({c for _, _, c in shapes}), "precision": args.precision,
        "l2": "inputs larger than L2 (126 MB), no flush",
        "parallelism": f"dp{world}" if world > 1 else "1 GPU",
    }


def run_domains(args, rank, world, local_rank):
    import ctypes as C

    import torch

    from more_benchmarks_dc_ocean_b200 import autotune, inputs
    from more_benchmarks_dc_ocean_b200 import ocean_redi as R

    # Inputs are generated before the first GPU call (the pool is spawned).
    workers = max(1, min(len(os.sched_getaffinity(0)), 8))  # host memory: one large domain per worker
    t_gen = time.perf_counter()
    ps = inputs.config4(seed=20261203 + 1000 * rank, n_domains=args.domains, workers=workers)
    t_gen = time.perf_counter() - t_gen
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist  # noqa: F811
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)
    dps = [R.to_device(p, dev) for p in ps]
    st = torch.cuda.current_stream()
    L = R.lib()
    L.redi_b200_launch_count.restype = C.c_ulonglong
    L.redi_b200_launch_count.argtypes = [C.c_int]
    prec_main = R.FP64 if args.precision == "fp64" else R.MIXED

    def reset_inputs():
        for p, dp in zip(ps, dps):
            dp.ms.h_layer.copy_(torch.from_numpy(p.h))
            for d, h in zip(dp.ms.tracers, p.tracers):
                d.copy_(torch.from_numpy(h))

    def barrier():
        if dist is not None:
            dist.barrier()

    def timed(batch, steps):
        barrier()
        torch.cuda.synchronize()
        L.redi_b200_profile_begin()
        n0 = L.redi_b200_launch_count(-1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        batch.step(steps, st)
        e1.record(st)
        torch.cuda.synchronize()
        n1 = L.redi_b200_launch_count(-1)
        kt = (C.c_double * NKERN)()
        kc = (C.c_ulonglong * NKERN)()
        L.redi_b200_profile_end(kt, kc, NKERN)
        barrier()
        return e0.elapsed_time(e1) / steps, kt, kc, int(n1 - n0)

    results = {}
    fp64_after_one = None
    for prec in ([R.FP64, R.MIXED] if prec_main == R.FP64 else [R.MIXED, R.FP64]):
        name = "fp64" if prec == R.FP64 else "mixed"
        reset_inputs()
        batch = R.RediBatch(dps, precision=prec)
        # One step from the initial state: FP64 is kept as the reference (bit-identical to the
        # oracle), the mixed result is compared with it domain by domain.
        batch.step(1, st)
        torch.cuda.synchronize()
        stat = batch.status()
        if prec == R.FP64:
            fp64_after_one = [[t.clone() for t in dp.ms.tracers] for dp in dps]
            err = None
        else:
            err = []
            if fp64_after_one is None:  # mixed ran first: make the FP64 reference now
                keep = [[t.clone() for t in dp.ms.tracers] for dp in dps]
                reset_inputs()
                ref_b = R.RediBatch(dps, precision=R.FP64)
                ref_b.step(1, st)
                torch.cuda.synchronize()
                fp64_after_one = [[t.clone() for t in dp.ms.tracers] for dp in dps]
                ref_b.destroy()
                for dp, k in zip(dps, keep):
                    for d, t in zip(dp.ms.tracers, k):
                        d.copy_(t)
                del keep
            for d, (dp, ref) in enumerate(zip(dps, fp64_after_one)):
                worst = 0.0
                for t, r in zip(dp.ms.tracers, ref):
                    worst = max(worst, float((t - r).abs().max()) / max(float(r.abs().max()), 1e-300))
                err.append(worst)
        tuning = None
        if not args.no_tune:
            tuning = autotune.tune_batch(batch, reps=2, stream=st)
            if dist is not None:
                t = torch.tensor(list(tuning["best"]), dtype=torch.int64, device=dev)
                dist.broadcast(t, 0)
                best = tuple(int(v) for v in t.tolist())
                batch.set_tuning(best[:2], best[2], best[3])
                tuning["best"] = best
        batch.step(args.warmup, st)
        torch.cuda.synchronize()
        clocks = ClockSampler(_uuid(local_rank)) if prec == prec_main else None
        if clocks:
            clocks.start()
        ms, kt, kc, launches = timed(batch, args.steps)
        clk = clocks.stop() if clocks else None
        batch.set_accounting(True)  # one more (untimed) step with per-stage accounting
        batch.step(1, st)
        stages = batch.stage_times()
        batch.set_accounting(False)
        ms_all = _max_over_ranks(ms, dist, dev)
        k = 8  # k_domain_persistent
        bytes_launch = float(sum(boundary_bytes(p, name) for p in ps))
        t_launch = kt[k] / max(1, kc[k]) * 1e-3
        results[name] = {
            "value": batch.updates * world / (ms_all * 1e-3), "ms_per_step": ms_all, "kernel_ms": kt[k] / max(1, kc[k]),
            "launches": launches, "bytes": bytes_launch, "achieved_gbs": bytes_launch / t_launch / 1e9,
            "status": stat, "clocks": clk, "updates": batch.updates, "items": batch.items,
            "stage_accounting_ms_summed_over_blocks": {k: {kk: round(vv, 3) if isinstance(vv, float) else vv
                                                           for kk, vv in v.items()} for k, v in stages.items()},
            "tuning": {"gather_tile": list(tuning["best"][:2]), "vertical_chunk": tuning["best"][2],
                       "occupancy": tuning["best"][3],
                       "grid_blocks": batch.get_tuning()["grid"], "candidates_ms": tuning["ms"]} if tuning else
            batch.get_tuning(),
            "per_domain_max_rel_err_vs_fp64_1step": ({"max": max(err), "median": statistics.median(err),
                                                      "all": [float(f"{e:.3e}") for e in err]} if err else None),
        }
        if prec == prec_main:
            results[name]["e2e"] = None if args.no_e2e else _domains_e2e(args, ps, dps, batch, st, dist, dev, world)
        batch.destroy()
        torch.cuda.synchronize()
    del fp64_after_one

    # Baseline on the same GPU: every domain stepped through the handle API, one after another.
    reset_inputs()
    handles = [R.make_redi(dp, prec_main) for dp in dps]
    for dp, h in zip(dps, handles):
        R.step(dp, h, args.warmup, st)
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n0 = L.redi_b200_launch_count(-1)
    L.redi_b200_profile_begin()
    e0.record(st)
    for _ in range(args.steps):
        for dp, h in zip(dps, handles):
            R.step(dp, h, 1, st)
    e1.record(st)
    torch.cuda.synchronize()
    skt = (C.c_double * NKERN)()
    skc = (C.c_ulonglong * NKERN)()
    L.redi_b200_profile_end(skt, skc, NKERN)
    seq_kernels = {KERNEL_NAMES[k]: round(skt[k] / args.steps, 3) for k in range(NKERN) if skc[k]}
    seq_launches = int(L.redi_b200_launch_count(-1) - n0) // args.steps
    seq_ms = _max_over_ranks(e0.elapsed_time(e1) / args.steps, dist, dev)
    for h in handles:
        h.destroy()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        big = max(ps, key=lambda p: p.ncell)
        upd, info = cpu_sample(big, args.cpu_seconds)
        cpu = {"value": upd, "unit": UNIT, "cores": info["cores"], "kind": "port", "sample": info["sample"]}

    main = results[args.precision]
    peak, peak_kind = _peaks()
    if rank == 0:
        line = {
            "metric": METRIC, "value": main["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": main["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f64+f32", "data": "synthetic",
            "config": _domains_config_block(ps, args, world, "plain FP64" if args.precision == "fp64" else "mixed"),
            "roofline": {"bound": "hbm", "kernel": "k_domain_persistent", "achieved": main["achieved_gbs"],
                         "peak": peak, "peak_source": peak_kind, "unit": "GB/s", "frac": main["achieved_gbs"] / peak,
                         "traffic": None, "algorithmic_bytes_per_launch": main["bytes"]},
            "side_by_side": {k: {kk: vv for kk, vv in v.items() if kk not in ("clocks", "e2e")}
                             for k, v in results.items()},
            "per_domain_launch_baseline": {"value": main["updates"] * world / (seq_ms * 1e-3), "ms_per_step": seq_ms,
                                           "launches_per_step": seq_launches, "kernel_ms_per_step": seq_kernels,
                                           "path": "handle API, one domain after another"},
            "cpu_baseline": cpu,
            "e2e": main["e2e"],
            "clocks": main["clocks"],
            "gpu_launches": main["launches"],
            "input_generation_s": round(t_gen, 1),
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def _domains_e2e(args, ps, dps, batch, st, dist, dev, world):
    import torch

    host = [(torch.from_numpy(p.h).pin_memory(), [torch.from_numpy(t).pin_memory() for t in p.tracers]) for p in ps]

    def e2e_step():
        for dp, (hh, ht) in zip(dps, host):
            dp.ms.h_layer.copy_(hh, non_blocking=True)
            for d, h in zip(dp.ms.tracers, ht):
                d.copy_(h, non_blocking=True)
        batch.step(1, st)
        for dp, (_, ht) in zip(dps, host):
            for d, h in zip(dp.ms.tracers, ht):
                h.copy_(d, non_blocking=True)

    for _ in range(max(1, args.warmup)):
        e2e_step()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(args.steps):
        e2e_step()
    e1.record(st)
    torch.cuda.synchronize()
    ms = _max_over_ranks(e0.elapsed_time(e1) / args.steps, dist, dev)
    cells = sum(p.nx * p.ny * p.nz for p in ps)
    ntr = ps[0].ntr
    return {"value": batch.updates * world / (ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": 8 * cells * (1 + ntr),
            "d2h_bytes_per_step": 8 * cells * ntr, "ms_per_step": ms, "host_memory": "pinned"}


def _uuid(local_rank):
    try:
        import torch

        u = str(torch.cuda.get_device_properties(local_rank).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        return None


def _max_over_ranks(x, dist, dev):
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _copy_floor_ms(host_h, host_tr, dp, st) -> float:
    """The e2e step's copies alone, with no kernels: h and every tracer up on one
    stream while every tracer comes down on another (separate buffers), best of
    3 after one warm-up. The bound the host-state step's pipeline can approach."""
    import torch

    up_dst = [torch.empty_like(dp.ms.h_layer)] + [torch.empty_like(d) for d in dp.ms.tracers]
    up_src = [host_h] + list(host_tr)
    down_dst = [torch.empty(t.shape, dtype=t.dtype, pin_memory=True) for t in host_tr]
    s_up, s_dn = torch.cuda.Stream(), torch.cuda.Stream()
    ts = []
    for _ in range(4):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        s_up.wait_event(a)
        s_dn.wait_event(a)
        with torch.cuda.stream(s_up):
            for d, h in zip(up_dst, up_src):
                d.copy_(h, non_blocking=True)
        with torch.cuda.stream(s_dn):
            for d, h in zip(dp.ms.tracers, down_dst):
                h.copy_(d, non_blocking=True)
        st.wait_stream(s_up)
        st.wait_stream(s_dn)
        b.record(st)
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    del up_dst, down_dst
    return min(ts[1:])


def _e2e(args, p, dp, redi, ex, st, dist, dev, world):
    import torch

    from more_benchmarks_dc_ocean_b200 import ocean_redi as R

    host_h = torch.from_numpy(np.ascontiguousarray(p.h)).pin_memory()
    host_tr = [torch.from_numpy(np.ascontiguousarray(t)).pin_memory() for t in p.tracers]
    path, bands, band_ms = "copies around the device entry points", None, None

    if ex is None:
        # One GPU: the host-state entry point, row bands pipelined through
        # upload / step / download streams.
        ms_host = R.MultilayerState(p.nz, host_h, host_tr, p.idx_temperature + 1, p.idx_salinity + 1)
        bands = 8

        def e2e_step():
            R.redi_step_host(dp.grid, dp.metrics, dp.eos, redi, ms_host, dp.dt, dp.khtr_u_ext, dp.khtr_v_ext,
                             dp.bc, bands, st)

        band_ms = {}
        for nb in (4, 8, 16, 32):  # pick the band count on the live problem (part of the warm-up)
            bands = nb
            e2e_step()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(st)
            e2e_step()
            b.record(st)
            torch.cuda.synchronize()
            band_ms[nb] = round(a.elapsed_time(b), 2)
        bands = min(band_ms, key=band_ms.get)
        path = f"redi_b200_step_host, {bands} row bands"
    else:
        def e2e_step():
            dp.ms.h_layer.copy_(host_h, non_blocking=True)
            for d, h in zip(dp.ms.tracers, host_tr):
                d.copy_(h, non_blocking=True)
            ex.exchange()
            R.step(dp, redi, 1, st)
            for d, h in zip(dp.ms.tracers, host_tr):
                h.copy_(d, non_blocking=True)

    for _ in range(max(1, args.warmup)):
        e2e_step()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(args.steps):
        e2e_step()
    e1.record(st)
    torch.cuda.synchronize()
    ms = _max_over_ranks(e0.elapsed_time(e1) / args.steps, dist, dev)
    nt = p.nx * p.ny * p.nz
    out = {"value": p.ntr * p.nx_phys * p.ny_phys * p.nz * world / (ms * 1e-3), "unit": UNIT,
           "h2d_bytes_per_step": 8 * nt * (1 + p.ntr), "d2h_bytes_per_step": 8 * nt * p.ntr, "ms_per_step": ms,
           "host_memory": "pinned", "path": path, "band_candidates_ms": band_ms}
    if ex is None:
        floor = _copy_floor_ms(host_h, host_tr, dp, st)
        out["copy_floor_ms"] = floor
        out["frac_of_copy_floor"] = floor / ms
    return out


# ---------------------------------------------------------------------------
# MEKE step (meke_step_ext): the diffusivity producer
# ---------------------------------------------------------------------------
MEKE_METRIC = "MEKE step column-steps/s (meke_step_ext, gabight_sph_meke_v100 configuration), 1 B200"
MEKE_UNIT = "column-steps/s"


def _meke_problem(config: str):
    from more_benchmarks_dc_ocean_b200 import meke_inputs as MI

    if config == "meke":  # the reference's benchmark: 473 x 297 points, 3 ghosts, 30 layers
        return MI.reference_ic()
    return MI.reference_ic(1440, 1080, 75, nghost=2)  # meke_c1: the Redi config-1 grid


def meke_bytes(nx: int, ny: int, nz: int):
    """Algorithmic bytes of the MEKE kernels per step at the gabight configuration (pass A, pass B).

    Pass A reads h and rho (nz layers each), areaT, meke, gm_src, ke_diss_ext, u_bbl2 and writes
    the zeroed SN faces, rd, ke_diss, depth, mass, 1/mass, both structure factors, Lmix, the source
    and the post-drag energy. Pass B reads the post-drag energy, mass, 1/area, 1/mass, the bottom
    factor, u_bbl2, the barotropic factor, Lmix and the four face metrics, and writes meke,
    kh_diff, ku and the two face fluxes."""
    nt, nu, nv = nx * ny, (nx + 1) * ny, nx * (ny + 1)
    a = 8 * (2 * nz * nt + 5 * nt + 10 * nt + nu + nv)
    b = 8 * (8 * nt + 2 * nu + 2 * nv + 3 * nt + nu + nv)
    return float(a), float(b)


def _ncu_traffic_tag(tag: str) -> dict:
    out = {}
    d = os.path.join(ROOT, "profiles")
    if not os.path.isdir(d):
        return out
    for fn in os.listdir(d):
        if fn.endswith(".md"):
            for line in open(os.path.join(d, fn)):
                m = re.match(rf"^traffic_bytes_per_launch_{tag}:\s*(\w+)\s*=\s*([\d.eE+]+)", line.strip())
                if m:
                    out[m.group(1)] = float(m.group(2))
    return out


def meke_cpu_sample(p, target_s: float, nsteps: int = 0, warmup: int = 0):
    """The MEKE oracle on the whole domain, all host threads; returns (column-steps/s, info)."""
    from oracle import meke_oracle as MO

    threads = len(os.sched_getaffinity(0))
    q = p.copy()
    t0 = time.perf_counter()
    MO.step(q, 1)
    probe = max(time.perf_counter() - t0, 1e-4)
    n = nsteps or int(max(3, min(400, target_s / probe)))
    times = []
    for s in range(warmup + n):
        t0 = time.perf_counter()
        MO.step(q, 1)
        if s >= warmup:
            times.append(time.perf_counter() - t0)
    t = min(times)
    return p.nx * p.ny / t, {"cores": threads, "t_step_s": t, "steps": n,
                             "sample": f"{p.nx}x{p.ny}x{p.nz} ({p.name}), whole domain, min of {n} step(s)"}


def _meke_config_block(p, world):
    return {"workload": f"MEKE step {p.nx}x{p.ny}x{p.nz} (arrays incl. ghosts), gabight_sph_meke_v100 "
                        f"(gmcoeff 0.9, khcoeff 1, cdrag 2.5e-3, kh 100)" + (f", {world} replicas" if world > 1 else ""),
            "grid": [p.nx, p.ny, p.nz], "dt_s": p.config["dt"],
            "l2": "L2 evicted before every timed step: 256 MB write, then 256 MB read (cold, clean L2)",
            "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"}


def run_meke_reference(args, rank, world):
    if rank != 0:
        return 0
    p = _meke_problem(args.config)
    budget = 120.0
    per = max(1.0, budget / max(1, args.steps + args.warmup))
    val, info = meke_cpu_sample(p, per, nsteps=args.steps, warmup=args.warmup)
    print(json.dumps({
        "impl": "reference", "metric": MEKE_METRIC, "value": val, "unit": MEKE_UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": info["t_step_s"] * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": _meke_config_block(p, world),
        "cpu_baseline": {"value": val, "unit": MEKE_UNIT, "cores": info["cores"], "kind": "port",
                         "sample": info["sample"]},
        "e2e": {"value": val, "unit": MEKE_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference CPU path (meke_step_ext restated in C++, OpenMP over all host cores); the Fortran "
                "build itself needs a Fortran compiler, absent on this image"}), flush=True)
    return 0


def run_meke(args, rank, world, local_rank):
    import ctypes as C

    import torch

    from more_benchmarks_dc_ocean_b200 import ocean_meke as M
    from more_benchmarks_dc_ocean_b200 import ocean_redi as R

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:  # independent replicas: the step has no exchange of its own
        import torch.distributed as dist  # noqa: F811
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)
    p = _meke_problem(args.config)
    d = M.to_device(p, dev)
    L = M.lib()
    RL = R.lib()
    RL.redi_b200_launch_count.restype = C.c_ulonglong
    RL.redi_b200_launch_count.argtypes = [C.c_int]
    h = C.c_void_p()
    assert L.meke_b200_create(p.nx, p.ny, p.nz, C.byref(h)) == 0, M.last_error()
    margs = M.make_args(p.nx, p.ny, p.nz, d, p.config)
    del2 = C.c_void_p(d["del2"].data_ptr())
    st = torch.cuda.current_stream()
    sp = C.c_void_p(st.cuda_stream)
    # L2 eviction between timed steps: a 256 MB write (twice the L2), then a 256 MB read that
    # writes those dirty lines back, so a timed step starts cold and inherits no write-back
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    clean = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    sink = torch.empty((), dtype=torch.float32, device=dev)

    def evict(i):
        flush.fill_(float(i))
        torch.sum(clean, dim=0, out=sink)

    def step():
        rc = L.meke_b200_step(h, C.byref(margs), del2, sp)
        if rc != 0:
            raise RuntimeError(M.last_error())

    def barrier():
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    def timed(nsteps, profile=False):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(nsteps)]
        if profile:
            RL.redi_b200_profile_begin()
        n0 = RL.redi_b200_launch_count(-1)
        for i in range(nsteps):
            evict(i)
            ev[i][0].record(st)
            step()
            ev[i][1].record(st)
        torch.cuda.synchronize()
        n1 = RL.redi_b200_launch_count(-1)
        kt = (C.c_double * NKERN)()
        kc = (C.c_ulonglong * NKERN)()
        if profile:
            RL.redi_b200_profile_end(kt, kc, NKERN)
        return sum(a.elapsed_time(b) for a, b in ev) / nsteps, int(n1 - n0), kt, kc

    clocks = ClockSampler(_uuid(local_rank))
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    ms, launches, _, _ = timed(args.steps)
    barrier()
    clk = clocks.stop()
    ms_all = _max_over_ranks(ms, dist, dev)
    value = p.nx * p.ny * world / (ms_all * 1e-3)

    # per-kernel device times (events around each launch: a separate pass, as they cut the programmatic edge)
    _, _, kt, kc = timed(args.steps, profile=True)
    kern = {KERNEL_NAMES[k]: {"ms_total": kt[k], "launches": int(kc[k]), "ms_per_launch": kt[k] / kc[k]}
            for k in range(NKERN) if kc[k]}
    bytes_a, bytes_b = meke_bytes(p.nx, p.ny, p.nz)
    peak, peak_kind = _peaks()
    ka, kb = 10, 12
    ta, tb = kt[ka] / kc[ka] * 1e-3, kt[kb] / kc[kb] * 1e-3
    achieved = bytes_a / ta / 1e9
    traffic = _ncu_traffic_tag("meke" if args.config == "meke" else "meke_c1").get("k_meke_column")

    # warm L2: back-to-back steps, no flush (the reference workload's fields fit in the 126 MB L2)
    w0, w1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0.record(st)
    for _ in range(args.steps):
        step()
    w1.record(st)
    torch.cuda.synchronize()
    warm_ms = w0.elapsed_time(w1) / args.steps

    e2e = None
    if not args.no_e2e:
        ins = ("h_layer", "rho_layer", "meke", "kh_diff", "gm_src", "ke_diss_ext", "u_bbl2")
        outs = ("meke", "kh_diff", "ku")
        host = {k: torch.from_numpy(np.ascontiguousarray(p.arrays[k])).pin_memory() for k in set(ins + outs)}

        def e2e_step():
            for k in ins:
                d[k].copy_(host[k], non_blocking=True)
            step()
            for k in outs:
                host[k].copy_(d[k], non_blocking=True)

        for _ in range(max(1, args.warmup)):
            e2e_step()
        torch.cuda.synchronize()
        barrier()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        for _ in range(args.steps):
            e2e_step()
        b.record(st)
        torch.cuda.synchronize()
        ems = _max_over_ranks(a.elapsed_time(b) / args.steps, dist, dev)
        e2e = {"value": p.nx * p.ny * world / (ems * 1e-3), "unit": MEKE_UNIT, "ms_per_step": ems,
               "h2d_bytes_per_step": int(sum(host[k].numel() * 8 for k in ins)),
               "d2h_bytes_per_step": int(sum(host[k].numel() * 8 for k in outs)), "host_memory": "pinned",
               "path": "meke_b200_step with its inputs copied up and meke / kh_diff / ku copied back every step"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, info = meke_cpu_sample(p, args.cpu_seconds)
        cpu = {"value": v, "unit": MEKE_UNIT, "cores": info["cores"], "kind": "port", "sample": info["sample"]}

    if rank == 0:
        print(json.dumps({
            "metric": MEKE_METRIC, "value": value, "unit": MEKE_UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_all, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": _meke_config_block(p, world),
            "roofline": {"bound": "hbm", "kernel": "k_meke_column", "achieved": achieved, "peak": peak,
                         "peak_source": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "algorithmic_bytes_per_launch": bytes_a},
            "step_roofline": {"algorithmic_bytes_per_step": bytes_a + bytes_b,
                              "achieved_gbs": (bytes_a + bytes_b) / (ms_all * 1e-3) / 1e9,
                              "frac": (bytes_a + bytes_b) / (ms_all * 1e-3) / 1e9 / peak,
                              "pass_b_gbs": bytes_b / tb / 1e9},
            "kernels": kern, "warm_l2_ms_per_step": warm_ms, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
            "gpu_launches": launches}), flush=True)
    L.meke_b200_destroy(h)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------
# ALE remap step (ale_remap_step): zstar target, PPM remap of T, S and the face velocities
# ---------------------------------------------------------------------------
ALE_METRIC = "ALE remap column-steps/s (ale_remap_step, zstar, PPM, T+S, face velocities), 1 B200"
ALE_UNIT = "column-steps/s"


def _ale_problem(config: str):
    from more_benchmarks_dc_ocean_b200 import ale_inputs as AI

    if config == "ale":  # the reference's benchmark: 473 x 297 points, 3 ghosts, 30 layers, h-drift 25 %
        return AI.reference_ic()
    return AI.reference_ic(1440, 1080, 75, nghost=2)  # ale_c1: the Redi config-1 grid


def ale_bytes(nx: int, ny: int, nz: int):
    """Algorithmic bytes of the ALE kernels per step (column tiles, face tiles), PPM, T and S.

    columns: read h, write h_old and target_h, read + write T, S, the heat, salt and mass budgets,
    write h_layer; faces: read h_old and target_h once, read + write u and v (2-D fields are
    negligible and not counted)."""
    n3, nu3, nv3 = nx * ny * nz, (nx + 1) * ny * nz, nx * (ny + 1) * nz
    return 8.0 * 14 * n3, 8.0 * (2 * n3 + 2 * nu3 + 2 * nv3)


def ale_cpu_sample(p, target_s: float, nsteps: int = 0, warmup: int = 0):
    from oracle import ale_oracle as AO

    threads = len(os.sched_getaffinity(0))
    q = p.copy()
    t0 = time.perf_counter()
    AO.step(q, 1)
    probe = max(time.perf_counter() - t0, 1e-4)
    n = nsteps or int(max(2, min(100, target_s / probe)))
    times = []
    for s in range(warmup + n):
        q = p.copy()  # from the pristine state, as the timed GPU steps
        t0 = time.perf_counter()
        AO.step(q, 1)
        if s >= warmup:
            times.append(time.perf_counter() - t0)
    t = min(times)
    return p.nx * p.ny / t, {"cores": threads, "t_step_s": t, "steps": n,
                             "sample": f"{p.nx}x{p.ny}x{p.nz} ({p.name}), whole domain from the pristine state, "
                                       f"min of {n} step(s)"}


def _ale_config_block(p, world):
    return {"workload": f"ALE remap {p.nx}x{p.ny}x{p.nz} (arrays incl. ghosts), zstar target, PPM, T+S with "
                        f"budgets, u/v face velocities, h-drift 25 %" + (f", {world} replicas" if world > 1 else ""),
            "grid": [p.nx, p.ny, p.nz],
            "l2": "state restored from the pristine copy, then L2 evicted (256 MB write + 256 MB read), before "
                  "every timed step",
            "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"}


def run_ale_reference(args, rank, world):
    if rank != 0:
        return 0
    p = _ale_problem(args.config)
    per = max(1.0, 120.0 / max(1, args.steps + args.warmup))
    val, info = ale_cpu_sample(p, per, nsteps=args.steps, warmup=args.warmup)
    print(json.dumps({
        "impl": "reference", "metric": ALE_METRIC, "value": val, "unit": ALE_UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": info["t_step_s"] * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": _ale_config_block(p, world),
        "cpu_baseline": {"value": val, "unit": ALE_UNIT, "cores": info["cores"], "kind": "port",
                         "sample": info["sample"]},
        "e2e": {"value": val, "unit": ALE_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference CPU path (ale_remap_step restated in C++, OpenMP over all host cores); the Fortran "
                "build itself needs a Fortran compiler, absent on this image"}), flush=True)
    return 0


def run_ale(args, rank, world, local_rank):
    import ctypes as C

    import torch

    from more_benchmarks_dc_ocean_b200 import ale_remap as A
    from more_benchmarks_dc_ocean_b200 import ocean_redi as R

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:  # independent replicas: the step has no exchange of its own
        import torch.distributed as dist  # noqa: F811
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)
    p = _ale_problem(args.config)
    d = A.to_device(p, dev)
    prist = {k: d[k].clone() for k in ("h_layer", "u", "v", "mass_budget", "heat_budget", "salt_budget", "bt_eta")}
    prist_tr = [t.clone() for t in d["tracers"]]
    RL = R.lib()
    RL.redi_b200_launch_count.restype = C.c_ulonglong
    RL.redi_b200_launch_count.argtypes = [C.c_int]
    st = torch.cuda.current_stream()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    clean = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    sink = torch.empty((), dtype=torch.float32, device=dev)

    def restore():
        for k, v in prist.items():
            d[k].copy_(v)
        for a, b in zip(d["tracers"], prist_tr):
            a.copy_(b)

    def evict(i):
        flush.fill_(float(i))
        torch.sum(clean, dim=0, out=sink)

    def step():
        A.step_problem(p, d, 1, st)

    def barrier():
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        restore()
        step()
    torch.cuda.synchronize()

    def timed(nsteps, profile=False):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(nsteps)]
        if profile:
            RL.redi_b200_profile_begin()
        n0 = RL.redi_b200_launch_count(-1)
        for i in range(nsteps):
            restore()
            evict(i)
            ev[i][0].record(st)
            step()
            ev[i][1].record(st)
        torch.cuda.synchronize()
        n1 = RL.redi_b200_launch_count(-1)
        kt = (C.c_double * NKERN)()
        kc = (C.c_ulonglong * NKERN)()
        if profile:
            RL.redi_b200_profile_end(kt, kc, NKERN)
        return sum(a.elapsed_time(b) for a, b in ev) / nsteps, int(n1 - n0), kt, kc

    clocks = ClockSampler(_uuid(local_rank))
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    ms, launches, _, _ = timed(args.steps)
    barrier()
    clk = clocks.stop()
    ms_all = _max_over_ranks(ms, dist, dev)
    value = p.nx * p.ny * world / (ms_all * 1e-3)
    _, _, kt, kc = timed(args.steps, profile=True)
    kern = {KERNEL_NAMES[k]: {"ms_total": kt[k], "launches": int(kc[k]), "ms_per_launch": kt[k] / kc[k]}
            for k in range(NKERN) if kc[k]}
    b_col, b_fc = ale_bytes(p.nx, p.ny, p.nz)
    kb = {13: b_col, 14: b_fc}
    top = max((k for k in kb if kc[k]), key=lambda k: kt[k])
    peak, peak_kind = _peaks()
    achieved = kb[top] / (kt[top] / kc[top] * 1e-3) / 1e9
    traffic = _ncu_traffic_tag("ale" if args.config == "ale" else "ale_c1").get(KERNEL_NAMES[top])
    total_b = b_col + b_fc

    e2e = None
    if not args.no_e2e:
        keys = ("h_layer", "u", "v", "mass_budget", "heat_budget", "salt_budget", "bt_eta")
        host = {k: prist[k].cpu().pin_memory() for k in keys}
        host_tr = [t.cpu().pin_memory() for t in prist_tr]

        def e2e_step():
            for k in keys:
                d[k].copy_(host[k], non_blocking=True)
            for a, b in zip(d["tracers"], host_tr):
                a.copy_(b, non_blocking=True)
            step()
            for k in keys:
                host[k].copy_(d[k], non_blocking=True)
            for a, b in zip(d["tracers"], host_tr):
                b.copy_(a, non_blocking=True)

        for _ in range(max(1, args.warmup)):
            e2e_step()
        torch.cuda.synchronize()
        barrier()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        for _ in range(args.steps):
            e2e_step()
        b.record(st)
        torch.cuda.synchronize()
        ems = _max_over_ranks(a.elapsed_time(b) / args.steps, dist, dev)
        nbytes = int(sum(host[k].numel() * 8 for k in keys) + sum(t.numel() * 8 for t in host_tr))
        e2e = {"value": p.nx * p.ny * world / (ems * 1e-3), "unit": ALE_UNIT, "ms_per_step": ems,
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes, "host_memory": "pinned",
               "path": "ale_b200_remap_step with the model state copied up and back every step"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, info = ale_cpu_sample(p, args.cpu_seconds)
        cpu = {"value": v, "unit": ALE_UNIT, "cores": info["cores"], "kind": "port", "sample": info["sample"]}

    if rank == 0:
        print(json.dumps({
            "metric": ALE_METRIC, "value": value, "unit": ALE_UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_all, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": _ale_config_block(p, world),
            "roofline": {"bound": "hbm", "kernel": KERNEL_NAMES[top], "achieved": achieved, "peak": peak,
                         "peak_source": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "algorithmic_bytes_per_launch": kb[top]},
            "step_roofline": {"algorithmic_bytes_per_step": total_b,
                              "achieved_gbs": total_b / (ms_all * 1e-3) / 1e9,
                              "frac": total_b / (ms_all * 1e-3) / 1e9 / peak},
            "kernels": kern, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk, "gpu_launches": launches}), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="config1",
                    choices=["config0", "config1", "config3", "config4", "meke", "meke_c1", "ale", "ale_c1"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--grid", default=None, help="NXxNYxNZ: a generated domain of that size instead of --config")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-sub", action="store_true", help="skip the mixed (config 2) and batched (config 3) sub-records")
    ap.add_argument("--fold", action="store_true",
                    help="Phase B as the fused face-flux + fold pass instead of the face-flux / cell-gather pair")
    ap.add_argument("--flux-staged", type=int, nargs="?", const=1, default=0, choices=(0, 1, 2),
                    help="face flux form: 1 the next sublayer's reconstruction staged through shared memory, "
                         "2 each column's reconstruction read through a two-layer shared-memory ring")
    ap.add_argument("--sweep-form", type=int, default=None, choices=(0, 3, 4, 5),
                    help="neutral sweep form: 0 register windows, 3/4/5 windows in a shared-memory ring")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-tune", action="store_true", help="skip the launch-shape autotuner")
    ap.add_argument("--domains", type=int, default=64, help="config4: number of regional domains")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    rank, world, local_rank = _rank_env()
    if args.impl == "reference":
        if args.config.startswith("meke"):
            return run_meke_reference(args, rank, world)
        if args.config.startswith("ale"):
            return run_ale_reference(args, rank, world)
        return run_reference(args, rank, world)
    if args.config.startswith("meke"):
        return run_meke(args, rank, world, local_rank)
    if args.config.startswith("ale"):
        return run_ale(args, rank, world, local_rank)
    if args.config == "config4":
        return run_domains(args, rank, world, local_rank)
    return run_b200(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
