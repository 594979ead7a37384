"""The non-headline configurations, measured for ``bench.py --workload ...``.

* ``li_rain_512``: local inertial, 512 x 512, dx 10 m, sloping plane + 20 seeded
  Gaussian bumps, n 0.03, uniform rain 50 mm/h for 3600 s (compensated), all edges
  open, alpha 0.7, the full 3600 s through run_simulation (device clock), plus the
  fused step kernel's roofline at the 40 B/cell-step it must move.
* ``li_reach_8192``: local inertial, 8192 x 8192, dx 5 m: a V-shaped valley with a
  down-valley slope and a meandering 3 m x 40 m channel, lognormal Manning
  (median 0.035, sigma 0.3), infiltration U(0, 20) mm/h, a triangular 500 m3/s
  hydrograph split over the 8 inlet channel cells, MPM bedload (d50 2 mm), open
  downstream edge; the first K steps (the full 12 h is ~10^5 steps), fused step
  roofline at 72 B/cell-step.
* ``li_rain_2048``: the rain-on-grid step at 2048 x 2048 (inputs larger than L2),
  the LI kernel's roofline point.
* ``hllc_lake_2048``: HLLC lake at rest, 2048 x 2048, dx 1 m, surface 2 m over
  seeded Gaussian bumps (amplitude 0.5-3.5 m, sigma 10-80 m) that pierce it, n 0.03,
  closed walls: the well-balanced case with dry islands and shorelines. Reports
  throughput and the largest |u|, |v| after the timed steps (round-off level).
* ``ensemble_256``: 256 local-inertial domains, sides log-uniform in [128, 2048],
  each with its own rain U(10, 100) mm/h and Manning U(0.02, 0.06), to 1800 s:
  the batched ensemble (autotuned tiles) against the plain per-domain loop
  (``compute_dt`` + ``step`` per step, one domain after another).
* ``serve``: Poisson request streams at each rate (sides 256-4096, horizons
  600-7200 s, 70 % LI / 30 % HLLC, 10 % Exner, 150 GB budget): solves/s and
  p50/p99 latency of the continuous-batching server against the serial loop.
All inputs are synthetic and seeded.
"""

from __future__ import annotations

import math
import statistics
import time

import numpy as np
import torch

import rbsim
from rbsim import _lib
from rbsim.config import Scenario
from rbsim.device_clock import DeviceClock
from rbsim.ensemble import Ensemble, autotune, log_uniform_sides
from rbsim.processes.inflow import Inflow, InflowInjector
from rbsim.sediment import arm_sediment


def _peak():
    import bench

    return bench.peaks()


# The float64-error leg (the CPU-baseline leg and the oracle helpers are in bench.py).
def _oracle():
    import bench

    return bench.oracle_module()


def _oracle_state(spec, dtype):
    import bench

    return bench.oracle_state(spec, dtype)


def cpu_leg(spec, **kw) -> dict:
    import bench

    return bench.cpu_leg(spec, **kw)


def _gpu_state(spec):
    from rbsim.schemes import hllc

    st = rbsim.State.from_bed(spec["bed"], spec["dx"], depth=spec["depth"], manning=spec["manning"])
    if spec["scheme"] == "hllc_fv":
        hllc.arm_hllc(st)
    if spec.get("infil") is not None:
        st.set_infiltration(spec["infil"])
    if spec.get("compensated"):
        st.arm_source_compensation()
    if spec.get("boundaries"):
        st.set_open_boundaries(spec["boundaries"])
    if spec.get("sediment"):
        arm_sediment(st, spec["sediment"]["d50"], spec["sediment"]["porosity"])
    inj = None
    if spec.get("inflows"):
        inj = InflowInjector([Inflow(tuple(c), list(h)) for c, h in spec["inflows"]], st.grid, st.device)
    return st, inj


def f64_leg(spec, steps: int) -> dict:
    """Error of the device's float32 result against the float64 oracle after ``steps``
    steps of ``spec``: the device steps through the public scheme API and records its
    timesteps; the float64 oracle replays them, so the runs differ only in precision."""
    o = _oracle()
    scheme = rbsim.get_scheme(spec["scheme"])
    st, inj = _gpu_state(spec)
    t, dts = 0.0, []
    for _ in range(steps):
        dt = scheme.compute_dt(st, alpha=spec["alpha"], dt_max=spec["dt_max"])
        if inj is not None:
            inj.apply(st, t, dt)
        scheme.step(st, dt=dt, rain=spec.get("rain", 0.0), t=t)
        dts.append(dt)
        t += dt
    qn = ("hu", "hv") if spec["scheme"] == "hllc_fv" else ("qx", "qy")
    got = {"h": st.h.cpu().numpy(), qn[0]: getattr(st, qn[0]).cpu().numpy(), qn[1]: getattr(st, qn[1]).cpu().numpy()}
    del st
    o.set_pow_mode(1)
    ref, rinj = _oracle_state(spec, np.float64)
    step = o.SCHEMES[spec["scheme"]][1]
    t = 0.0
    for dt in dts:
        if rinj is not None:
            rinj.apply(ref, t, dt)
        step(ref, dt, rain=spec.get("rain", 0.0))
        t += dt
    o.set_pow_mode(0)
    h64 = ref.h
    h_max = float(np.abs(h64).max())
    q_scale = max([float(np.abs(getattr(ref, k)).max()) for k in qn] + [h_max * math.sqrt(9.81 * h_max)])
    dq = max(float(np.abs(got[k].astype(np.float64) - getattr(ref, k)).max()) for k in qn)
    dh = float(np.abs(got["h"].astype(np.float64) - h64).max())
    v64 = float(h64.sum())
    return {"steps": steps, "max_abs_depth_m": dh, "max_rel_depth": dh / h_max if h_max > 0 else 0.0,
            "max_abs_discharge_m2_s": dq, "max_rel_discharge": dq / q_scale if q_scale > 0 else 0.0,
            "rel_volume": abs(float(got["h"].astype(np.float64).sum()) - v64) / v64 if v64 > 0 else 0.0,
            "reference": "float64 build of the same kernels (oracle/librbo_f64.so), replaying the device's "
                         "timesteps; discharge relative to max(|q|_max, h_max sqrt(g h_max))"}  # fmt: skip


def _bumps(ny, nx, dx, rng, n, amp, sigma, slope=1e-3):
    yy, xx = np.mgrid[0:ny, 0:nx].astype(np.float32)
    z = slope * xx * dx
    for _ in range(n):
        a, s = rng.uniform(*amp), rng.uniform(*sigma)
        cy, cx = rng.uniform(0, ny), rng.uniform(0, nx)
        z += a * np.exp(-((yy - cy) ** 2 + (xx - cx) ** 2) * dx * dx / (2 * s * s))
    return z.astype(np.float32)


def _kernel_roofline(state, scheme, steps, bytes_per_cell, injector=None, rain_rate=0.0):
    """Per-launch CUDA-event time of the step kernel(s) over a timed span of device-clock steps."""
    import ctypes

    L = _lib.lib()
    clk = DeviceClock(state, scheme, alpha=0.7, dt_max=30.0, sync_times=[1e9], graph_steps=steps,
                      injector=injector, rain_rate=rain_rate, rain_until=1e9)  # fmt: skip
    f = state.li_fields()
    ws = state.workspace.data_ptr()
    stream = torch.cuda.current_stream()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    clk.set_target(1e9, steps)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    for k in range(steps):
        _lib.check(L.rb_clock_plan(ws, stream.cuda_stream))
        if injector is not None:
            _lib.check(L.rb_clock_inflow(state._h.bufs[0].data_ptr(), state._h.bufs[1].data_ptr(), ws,
                                         stream.cuda_stream))  # fmt: skip
        ev[k][0].record()
        _lib.check(L.rb_li_step_clocked(ctypes.byref(f), ws, stream.cuda_stream))
        ev[k][1].record()
    stop.record()
    torch.cuda.synchronize()
    clk.read()
    cells = state.grid.n_cells
    kms = statistics.mean(a.elapsed_time(b) for a, b in ev)
    achieved = bytes_per_cell * cells / (kms / 1e3) / 1e9
    pk = _peak()
    return {
        "bound": "hbm", "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
        "frac": achieved / pk["hbm_gbs"], "traffic": None, "peak_source": pk["source"],
        "kernel": "li_step_kernel", "kernel_ms_mean": kms, "bytes_per_cell_step": bytes_per_cell,
        "gcell_per_s_kernel": cells / (kms / 1e3) / 1e9,
        "gcell_per_s_step": cells * steps / (start.elapsed_time(stop) / 1e3) / 1e9,
        "timed_s": start.elapsed_time(stop) / 1e3, "cell_updates": cells * steps,
    }  # fmt: skip


def li_rain_512(args):
    from rbsim.run import run_simulation

    n, dx = 512, 10.0
    rng = np.random.default_rng(1)
    bed = _bumps(n, n, dx, rng, 20, (0.5, 5.0), (50.0, 300.0))
    sc = Scenario(name="li_rain_512", scheme="local_inertial", dx=dx, end_time=3600.0, output_every=600.0,
                  alpha=0.7, dt_max=30.0, rain_mm_hr=50.0, rain_duration=3600.0, manning=0.03,
                  boundaries={e: "open" for e in ("north", "south", "east", "west")}, bed=bed)  # fmt: skip
    import tempfile

    with tempfile.TemporaryDirectory() as tmp:
        run_simulation(sc, None, f"{tmp}/warm.zarr", verbose=False)  # build + warm
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ledger = run_simulation(sc, None, f"{tmp}/r.zarr", verbose=False)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    st = rbsim.State.from_bed(bed, dx, depth=0.05, manning=0.03)
    st.arm_source_compensation()
    st.set_open_boundaries({e: "open" for e in ("north", "south", "east", "west")})
    roof = _kernel_roofline(st, "local_inertial", 200, 40)
    return {"workload": "li_rain_512", "metric": "Gcell-updates/s", "full_run_wall_s": wall,
            "mass_max_rel_error": ledger.max_rel_error, "roofline": roof}  # fmt: skip


RAIN_50_MM_H = 50.0 / 1000.0 / 3600.0


def li_rain_2048_spec() -> dict:
    """Rain-on-grid at 2048^2, dx 10 m: a sloping bed with 40 Gaussian bumps, 0.5-0.6 m of
    water, n 0.03, compensated uniform rain 50 mm/h, every edge open."""
    n, dx = 2048, 10.0
    rng = np.random.default_rng(1)
    bed = _bumps(n, n, dx, rng, 40, (0.5, 5.0), (50.0, 1200.0))
    return dict(scheme="local_inertial", bed=bed, dx=dx, depth=(0.5 + 0.1 * rng.random((n, n))).astype(np.float32),
                manning=0.03, compensated=True, rain=RAIN_50_MM_H,
                boundaries={e: "open" for e in ("north", "south", "east", "west")}, alpha=0.7, dt_max=30.0)  # fmt: skip


def li_rain_2048(args, legs: bool = True):
    """The rain-on-grid step at 2048^2 (inputs larger than L2): the LI kernel's roofline
    point, 40 algorithmic bytes per cell-step (read h, z, n, qx, qy, h_comp; write h, qx,
    qy, h_comp); with ``legs``, the CPU oracle on the same grid and the float64 error."""
    spec = li_rain_2048_spec()
    st, _ = _gpu_state(spec)
    _kernel_roofline(st, "local_inertial", max(args.warmup, 1), 40, rain_rate=RAIN_50_MM_H)  # warm-up steps
    roof = _kernel_roofline(st, "local_inertial", args.steps, 40, rain_rate=RAIN_50_MM_H)
    # DRAM bytes read + written by one launch in an ncu capture of this workload (fast
    # build): 100.8 + 30.9 MB against 167.8 MB algorithmic (L2 keeps part of the last step)
    roof["traffic"] = 131.6e6
    roof["traffic_note"] = "one launch, ncu --set full capture of this workload (fast build)"
    del st
    out = {"workload": "li_rain_2048", "metric": "Gcell-updates/s", "value": roof["gcell_per_s_step"],
           "steps": args.steps, "warmup": args.warmup, "roofline": roof,
           "config": {"grid": [2048, 2048], "dx_m": 10.0, "rain_mm_h": 50.0, "edges": "open", "manning": 0.03,
                      "l2": "9 float32 fields of 16.8 MB touched per step (151 MB) vs 126 MB L2"}}  # fmt: skip
    if legs:
        cpu = cpu_leg(spec, budget_s=8.0)
        cpu["sample"] = f"{cpu['steps']} steps of the full 2048 x 2048 grid, C oracle with OpenMP"
        out["cpu_baseline"] = cpu
        out["err_vs_f64"] = f64_leg(spec, steps=20)
    return out


def hllc_lake_2048(args):
    from rbsim.schemes import hllc

    n, dx = 2048, 1.0
    rng = np.random.default_rng(2)
    bed = _bumps(n, n, dx, rng, 40, (0.5, 3.5), (10.0, 80.0), slope=0.0)
    depth = np.maximum(2.0 - bed, 0.0).astype(np.float32)
    st = rbsim.State.from_bed(bed, dx, depth=depth, manning=0.03)
    hllc.arm_hllc(st)
    v0 = st.volume_sum()
    K = args.steps
    clk = DeviceClock(st, "hllc_fv", alpha=0.45, dt_max=30.0, sync_times=[600.0], graph_steps=K)
    clk.run_until(600.0, max_steps=K)  # capture + warm
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clk.set_target(600.0, K)
    start.record()
    clk._replay()
    stop.record()
    torch.cuda.synchronize()
    clk.read()
    ms = start.elapsed_time(stop) / K

    def at_rest():
        u, v = st.velocities_numpy()
        h = st.h.cpu().numpy()
        speed = np.maximum(np.abs(u), np.abs(v))
        deep = h > 0.1
        return {"t_s": clk.t, "steps": clk.steps, "max_speed": float(speed.max()),
                "max_speed_where_deeper_than_0.1m": float(speed[deep].max()) if deep.any() else 0.0,
                "volume_rel_change": abs(st.volume_sum() - v0) / v0}  # fmt: skip

    after_timed = at_rest()
    # then on to the configuration's 600 s horizon (untimed), where its gate is read
    clk.run_until(600.0)
    horizon = at_rest()
    h = st.h.cpu().numpy()
    return {"workload": "hllc_lake_2048", "metric": "Gcell-updates/s", "value": n * n / (ms / 1e3) / 1e9,
            "ms_per_step": ms, "steps": K, "dry_fraction": float((h < 1e-3).mean()),
            "after_timed_steps": after_timed, "at_600s": horizon}  # fmt: skip


def reach_inputs(n=8192, dx=5.0, seed=3):
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:n, 0:n].astype(np.float32)
    centre = n / 2 + (400.0 / dx) * np.sin(2 * np.pi * xx * dx / 3000.0)
    dist = np.abs(yy - centre) * dx
    z = 0.05 * dist + 1e-3 * (n - 1 - xx) * dx
    chan = dist <= 20.0
    z = np.where(chan, z - 3.0, z).astype(np.float32)
    manning = np.exp(np.log(0.035) + 0.3 * rng.standard_normal((n, n))).astype(np.float32)
    infil = (rng.uniform(0.0, 20.0, (n, n)) / 1000.0 / 3600.0).astype(np.float32)
    inlet_rows = np.nonzero(chan[:, 0])[0][:8]
    hydro = [(0.0, 0.0), (7200.0, 500.0 / len(inlet_rows)), (14400.0, 0.0)]
    inflows = [Inflow((int(r), 0), hydro) for r in inlet_rows]
    depth = np.where(chan, 2.0, 0.05).astype(np.float32)  # a wet valley: every face path is exercised
    return z, manning, infil, inflows, depth


def reach_band_spec(z, manning, infil, inflows, depth, rows: int) -> dict:
    """Rows n/2 - rows/2 .. n/2 + rows/2 - 1 of the reach: the meandering channel and all
    eight inflow cells lie inside; bedload armed (no Exner activation in so few steps)."""
    n = z.shape[1]
    r0 = z.shape[0] // 2 - rows // 2
    band = slice(r0, r0 + rows)
    return dict(scheme="local_inertial", bed=z[band].copy(), dx=5.0, depth=depth[band].copy(),
                manning=manning[band].copy(), infil=infil[band].copy(),
                inflows=[((inf.cell[0] - r0, inf.cell[1]), inf.hydrograph) for inf in inflows],
                boundaries={"east": "open"}, sediment=dict(d50=np.full((rows, n), 0.002, np.float32), porosity=0.4),
                alpha=0.7, dt_max=30.0)  # fmt: skip


def li_reach_8192(args, legs: bool = True):
    """The largest single-GPU configuration: the 8192^2 valley reach (infiltration, eight
    inflow cells, bedload), 72 algorithmic bytes per cell-step; with ``legs``, the CPU
    oracle and the float64 error on a 512 x 8192 band of it."""
    n, dx = 8192, 5.0
    z, manning, infil, inflows, depth = reach_inputs(n, dx)
    st = rbsim.State.from_bed(z, dx, depth=depth, manning=manning)
    st.set_infiltration(infil)
    st.set_open_boundaries({"east": "open"})
    arm_sediment(st, 0.002, 0.4)
    inj = InflowInjector(inflows, st.grid, st.device)
    # warm up on the first steps of the flood so transport is active, then time
    clk = DeviceClock(st, "local_inertial", alpha=0.7, dt_max=30.0, sync_times=[43200.0],
                      graph_steps=max(args.warmup, 1), injector=inj)  # fmt: skip
    clk.run_until(43200.0, max_steps=max(args.warmup, 1))
    clk.close()
    roof = _kernel_roofline(st, "local_inertial", args.steps, 72, injector=inj)
    del st, clk, inj
    torch.cuda.empty_cache()
    out = {"workload": "li_reach_8192", "metric": "Gcell-updates/s", "value": roof["gcell_per_s_step"],
           "steps": args.steps, "warmup": args.warmup, "roofline": roof,
           "config": {"grid": [n, n], "dx_m": dx, "inflow_cells": len(inflows), "edges": "east open",
                      "physics": "infiltration U(0, 20) mm/h, lognormal Manning (median 0.035, sigma 0.3), "
                                 "MPM bedload d50 2 mm"}}  # fmt: skip
    if legs:
        spec = reach_band_spec(z, manning, infil, inflows, depth, rows=512)
        cpu = cpu_leg(spec, budget_s=8.0)
        cpu["sample"] = f"{cpu['steps']} steps of a 512 x 8192 band of the reach (the channel and the inflows), " \
                        "C oracle with OpenMP"
        out["cpu_baseline"] = cpu
        out["err_vs_f64"] = f64_leg(spec, steps=10)
        out["err_vs_f64"]["sample"] = "the same 512 x 8192 band"
    return out


def _digest(t: torch.Tensor) -> str:
    import hashlib

    return hashlib.blake2b(t.cpu().numpy().tobytes(), digest_size=16).hexdigest()


def _ensemble_members(n=256, seed=5):
    rng = np.random.default_rng(seed)
    sides = log_uniform_sides(n, 128, 2048, seed)
    out = []
    for k, side in enumerate(sides):
        bed = _bumps(side, side, 10.0, np.random.default_rng(1000 + k), 8, (0.5, 3.0), (30.0, 0.15 * side * 10.0))
        out.append((bed, float(rng.uniform(10.0, 100.0)) / 3.6e6, float(rng.uniform(0.02, 0.06))))
    return out


def _ensemble_vs_plain(spec, horizon: float) -> dict:
    """``spec`` (bed, rain, Manning per domain) to ``horizon``: the plain per-domain loop,
    then the batched ensemble from fresh states; wall times, steps and the digests."""
    from rbsim.scheduler import MultiRateScheduler
    from rbsim.schemes import local_inertial as li

    def fresh():
        sts = []
        for bed, _, n_ in spec:
            st = rbsim.State.from_bed(bed, 10.0, depth=0.0, manning=n_)
            st.arm_source_compensation()
            sts.append(st)
        return sts

    # plain loop: each domain to the horizon through compute_dt + step, one after another
    sts = fresh()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plain_steps = []
    for st, (_, rain, _) in zip(sts, spec, strict=True):
        sched = MultiRateScheduler(end_time=horizon, output_every=horizon)
        k = 0
        for tick in sched.ticks(lambda st=st: li.compute_dt(st, 0.7, 30.0)):
            li.step(st, tick.dt, rain=rain)
            k += 1
        plain_steps.append(k)
    torch.cuda.synchronize()
    plain_wall = time.perf_counter() - t0
    plain_h = [_digest(st.h) for st in sts]  # every member's final depth, as a digest
    del sts
    torch.cuda.empty_cache()

    sts = fresh()
    rains = [r for _, r, _ in spec]

    def make(li_v, hl_v, t_start, graph_steps=8):
        e = Ensemble(sts, ["local_inertial"] * len(sts), alpha=0.7, dt_max=30.0, sync_times=[[horizon]] * len(sts),
                     rain_rate=rains, rain_until=[horizon] * len(sts), li_variant=li_v, hllc_variant=hl_v,
                     graph_steps=graph_steps, t0=0.0 if t_start is None else t_start)  # fmt: skip
        e.set_targets(horizon)
        return e

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    # the probe replays are real steps of the run; the batch continues from where they stopped
    best, timings, t_reached = autotune(make, probe_replays=1, candidates=[(0, 0), (1, 0), (2, 0), (3, 0)])
    ens = make(*best, t_reached, graph_steps=32)
    replays = ens.run_until(horizon)
    torch.cuda.synchronize()
    batched_wall = time.perf_counter() - t0
    same = sum(_digest(st.h) == d for st, d in zip(sts, plain_h, strict=True))
    steps = [c.steps for c in ens.clock]
    cell_updates = sum(k * b.size for k, (b, _, _) in zip(steps, spec, strict=True))
    del ens, sts
    torch.cuda.empty_cache()
    return {"batched_wall": batched_wall, "plain_wall": plain_wall, "replays": replays, "best": best,
            "timings": timings, "steps": steps, "plain_steps": plain_steps, "same": same,
            "cell_updates": cell_updates}  # fmt: skip


def _host_step_overhead(samples: int = 300) -> float:
    """Seconds the plain loop spends per step outside the kernel: compute_dt (a reduction
    and a read-back) + step on a domain small enough that the kernels cost nothing."""
    from rbsim.schemes import local_inertial as li

    st = rbsim.State.from_bed(np.zeros((32, 32), np.float32), 10.0, depth=0.1, manning=0.03)
    st.arm_source_compensation()
    for _ in range(20):
        li.step(st, li.compute_dt(st, 0.7, 30.0), rain=1e-5)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(samples):
        li.step(st, li.compute_dt(st, 0.7, 30.0), rain=1e-5)
    torch.cuda.synchronize()
    return (time.perf_counter() - t0) / samples


def ensemble_256(args):
    """Config 4. Under torchrun each rank takes its share of the 256 domains (whole
    domains, longest first onto the least-loaded rank); solves/s is all domains over
    the slowest rank's time.

    Also measured: the small-domain share (sides <= 512) on its own, and the bound on
    batched / plain that the kernel rate allows. The batched run cannot step faster
    than its kernel rate R (cell-updates/s), and the plain loop pays, per step, the
    kernel time plus a host overhead t_host (the dt read-back and the launch), so
    plain / batched <= sum_d steps_d (cells_d / R + t_host) / sum_d steps_d cells_d / R."""
    from rbsim import replicas

    horizon = 1800.0
    rank, world = replicas.rank_world()
    all_spec = _ensemble_members()
    mine = replicas.shard_units([float(b.size) for b, _, _ in all_spec], world)[rank]
    spec = [all_spec[i] for i in mine]
    cells = sum(b.size for b, _, _ in spec)
    t_host = _host_step_overhead()

    def record(r, sub):
        job_rate, job_wall = replicas.whole_job_rate(float(len(sub)), r["batched_wall"])
        plain_rate, plain_job_wall = replicas.whole_job_rate(float(len(sub)), r["plain_wall"])
        rate = r["cell_updates"] / r["batched_wall"]
        work = sum(k * b.size for k, (b, _, _) in zip(r["plain_steps"], sub, strict=True))
        bound = (work / rate + t_host * sum(r["plain_steps"])) / (work / rate)
        return {
            "domains": len(sub), "cells": sum(b.size for b, _, _ in sub),
            "batched": {"wall_s": job_wall, "solves_per_s": job_rate, "replays": r["replays"],
                        "tiles": {"li_variant": r["best"][0]},
                        "autotune_ms_per_replay": {str(k): v for k, v in r["timings"].items()},
                        "gcell_per_s_this_rank": rate / 1e9, "steps": sum(r["steps"])},
            "plain_loop": {"wall_s": plain_job_wall, "solves_per_s": plain_rate, "steps": sum(r["plain_steps"])},
            "speedup": plain_job_wall / job_wall,
            "speedup_bound_at_this_kernel_rate": bound,
            "domains_bitwise_equal_to_plain": f"{r['same']} of {len(sub)}",
            "all_domains_bitwise_equal_to_plain": r["same"] == len(sub),
        }  # fmt: skip

    full = record(_ensemble_vs_plain(spec, horizon), spec)
    small = [m for m in spec if m[0].shape[0] <= 512]
    out = {"workload": "ensemble_256", "metric": "ensemble solves/s", "n_gpus": world, "domains": len(all_spec),
           "domains_this_rank": len(spec), "cells_this_rank": cells, "host_overhead_per_plain_step_s": t_host,
           **full}  # fmt: skip
    if small:
        out["small_domains_up_to_512"] = record(_ensemble_vs_plain(small, horizon), small)
    return out


def serve(args):
    import tempfile

    from rbsim.serve import Server, poisson_stream, serial_baseline, serial_per_step_baseline

    out = {"workload": "serve", "metric": "solves/s, p50/p99 latency", "rates": {},
           "frames": "every request streams a frame every 600 simulated s and at its horizon to its own result "
                     "store, in both the batched server and the serial loop"}  # fmt: skip
    for rate in [float(r) for r in args.rates.split(",") if r.strip() and r.strip() != "none"]:
        reqs = poisson_stream(rate, args.requests, seed=int(rate * 100))
        for r in reqs:
            r.output_every = 600.0
        with tempfile.TemporaryDirectory() as tmp:
            srv = Server(hbm_budget=150e9, graph_steps=16, out_dir=f"{tmp}/batched")
            srv.run(reqs)
            torch.cuda.empty_cache()
            serial = serial_baseline(reqs, out_dir=f"{tmp}/serial")
        out["rates"][str(rate)] = {"batched": srv.stats, "serial": serial,
                                   "throughput_ratio": srv.stats["solves_per_s"] / serial["solves_per_s"]}  # fmt: skip
        torch.cuda.empty_cache()
    # the small-request share on its own: sides 256-512, where the serial loop is launch-bound;
    # a stream long enough (8 x --requests) that the batch reaches a steady state instead of
    # waiting on its one longest request
    reqs = poisson_stream(50.0, 8 * args.requests, seed=4242, side_lo=256, side_hi=512)
    with tempfile.TemporaryDirectory() as tmp:
        for r in reqs:
            r.output_every = 600.0
        srv = Server(hbm_budget=150e9, graph_steps=16, out_dir=f"{tmp}/batched")
        srv.run(reqs)
        torch.cuda.empty_cache()
        serial = serial_baseline(reqs, out_dir=f"{tmp}/serial")
        per_step = serial_per_step_baseline(reqs, out_dir=f"{tmp}/per_step")
    out["small_requests_256_512_at_50_per_s"] = {"requests": len(reqs),
        "batched": srv.stats, "serial": serial, "serial_per_step": per_step,
        "throughput_ratio": srv.stats["solves_per_s"] / serial["solves_per_s"],
        "throughput_ratio_vs_per_step_loop": srv.stats["solves_per_s"] / per_step["solves_per_s"],
        "baselines": "serial: each request alone on the device clock (graph-replayed spans); serial_per_step: "
                     "each request alone through compute_dt + step per step, the reference's loop"}  # fmt: skip
    return out


def run(args):
    """Run one workload. Under torchrun (WORLD_SIZE > 1) each rank drives its own GPU
    and the workloads that shard (ensemble_256) split their units across ranks; the
    others run one replica per rank."""
    import os

    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    fn = {"li_rain_512": li_rain_512, "li_rain_2048": li_rain_2048, "hllc_lake_2048": hllc_lake_2048,
          "li_reach_8192": li_reach_8192, "ensemble_256": ensemble_256, "serve": serve}[args.workload]  # fmt: skip
    from rbsim import arith

    # ensembles run the exact arithmetic, so their plain-loop comparisons do too
    mode = "exact" if args.workload in ("ensemble_256", "serve") else args.arith
    arith.set_arithmetic(mode)
    try:
        if args.workload in ("li_rain_2048", "li_reach_8192"):
            out = fn(args, legs=not args.no_legs)
        else:
            out = fn(args)
        out["build"] = mode
        return out
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
