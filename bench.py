"""Benchmark of the solver hot path on B200: Gcell-updates/s of the HLLC step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl rbsim|reference]

Workload (the headline configuration): HLLC well-balanced 2D, 2048 x 2048 float32,
dx = 1 m, dam break on a flat frictionless bed (h = 10 m for x < 1024, 1 m beyond,
at rest), closed walls, alpha = 0.45. One "step" = the CFL reduction + one SSP-RK2
step (both Heun stages with friction and sources). Synthetic inputs, generated
here.

* ``value``: whole-job cell-updates per second with the state resident on the
  device: K steps on the device-resident clock (dt, fill_span and rain gating in
  a one-thread plan kernel), replayed as one CUDA graph, timed with CUDA events
  between a barrier + synchronize on each side (max over ranks).
* ``e2e``: the same metric through the public API from host memory: the bed and
  initial depth are copied in from pinned host buffers (State.from_bed), K steps
  run through DeviceClock, and the final depth is copied back to a pinned buffer,
  all inside the timed region. ``e2e.per_step_api`` is the same through the
  reference-shaped ``compute_dt`` / ``step`` loop, which reads dt back to the host
  every step as the reference does.
* ``roofline``: the step's kernels against the measured HBM copy bandwidth, from
  algorithmic bytes (32 B per cell-step: read h, hu, hv, z, n; write h, hu, hv) over
  the CUDA-event time of the timed replay itself (which also holds the one-thread
  plan kernel of each step, so the figure is a lower bound for the stage pair);
  ``launched_one_by_one`` times each stage kernel with events around single launches
  as a cross-check.
* ``cpu_baseline``: the CPU oracle (the reference's kernels restated in C, OpenMP
  over the host cores, libm powf) on the full 2048 x 2048 grid for ~10 s.
* ``err_vs_f64``: the device result after 12 steps against the float64 build of the
  same kernels replaying the device's timesteps.
* ``workloads``: the LI roofline point (2048^2 rain-on-grid, 40 B/cell-step) and the
  largest single-GPU configuration (the 8192^2 valley reach, 72 B/cell-step), each
  with its own roofline, CPU baseline and float64 error.

Under torchrun each rank runs an independent replica of the workload on its own
GPU (replicas only: the path has no exchange step), ``scaling`` = "weak".
``--impl reference`` times the CPU oracle port of the reference path on the same
2048 x 2048 grid, W warm-up steps then K timed steps (rank 0 alone).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "river-basin-sim_b200"))

import numpy as np  # noqa: E402

N = 2048
DX = 1.0
ALPHA = 0.45
DT_MAX = 30.0
T_END = 30.0  # simulated horizon of the dam-break configuration
BYTES_PER_CELL_STEP = 32  # read h, hu, hv, z, n (20 B) + write h, hu, hv (12 B)
# DRAM bytes (read + write) of one step's two stage launches in one ncu capture of this
# workload (--set full, 2048^2 dam break, fast build, stage 1 + stage 2): 87.2 MB +
# 165.5 MB (the exact build: 88.3 + 163.5 MB).
NCU_DRAM_BYTES_PER_STEP = 252.7e6
# The stage kernels are issue-bound: share of issue slots busy in the same capture
# (fast build: stage 1 83.4 %, stage 2 82.4 %; exact: 84.8 %, 84.3 %).
NCU_ISSUE_ACTIVE = (0.834, 0.824)
WORKLOAD = "hllc_dambreak_2048x2048"
BUILDS = {
    "exact": "exact: one IEEE rounding per operation in the reference's order, bit-identical to the oracle",
    "fast": "fast: contracted multiply-adds, approximate division / square root / powers; within 1e-5 relative "
            "(L2) and 1e-4 m of the oracle on the same timesteps, every physics gate",
}


def dambreak_inputs(n: int = N):
    depth = np.ones((n, n), np.float32)
    depth[:, : n // 2] = 10.0
    return np.zeros((n, n), np.float32), depth


def peaks() -> dict:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        if self.index < 0:  # sampling off
            return self
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)  # fmt: skip
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) != 6:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[2:], strict=True):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": max(mx) if mx else None,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


# --------------------------------------------------------------------------- #
# CPU-baseline leg and the oracle helpers the float64-error leg shares. The    #
# oracle (oracle/: the reference's kernels restated in C) is the checker and   #
# the CPU baseline: it is timed beside the device path and compared with it,   #
# never part of what is measured on the device.                                #
# --------------------------------------------------------------------------- #
def oracle_module():
    here = os.path.join(ROOT, "oracle")
    if here not in sys.path:
        sys.path.insert(0, here)
    import oracle

    return oracle


def oracle_state(spec, dtype):
    o = oracle_module()
    st = o.State.from_bed(spec["bed"], spec["dx"], depth=spec["depth"], manning=spec["manning"], dtype=dtype)
    if spec["scheme"] == "hllc_fv":
        st.arm_hllc()
    if spec.get("infil") is not None:
        st.set_infiltration(spec["infil"])
    if spec.get("compensated"):
        st.arm_source_compensation()
    if spec.get("boundaries"):
        st.set_open_boundaries(spec["boundaries"])
    if spec.get("sediment"):
        st.arm_sediment(spec["sediment"]["d50"], spec["sediment"]["porosity"])
    inj = None
    if spec.get("inflows"):
        inj = o.InflowInjector([o.Inflow(tuple(c), list(h)) for c, h in spec["inflows"]], st.ny, st.nx, st.dx)
    return st, inj


def cpu_leg(spec, *, budget_s=10.0, steps_cap=1000, warmup=1, pow_mode=0) -> dict:
    """The CPU oracle stepping ``spec`` (compute_dt + sources + step) for at most
    ``budget_s`` seconds after ``warmup`` untimed steps; OpenMP over the host's cores."""
    o = oracle_module()
    o.set_pow_mode(pow_mode)
    st, inj = oracle_state(spec, np.float32)
    cdt, step = o.SCHEMES[spec["scheme"]]
    t, steps = 0.0, 0

    def one():
        nonlocal t
        dt = cdt(st, spec["alpha"], spec["dt_max"])
        if inj is not None:
            inj.apply(st, t, dt)
        step(st, dt, rain=spec.get("rain", 0.0))
        t += dt

    for _ in range(warmup):
        one()
    t0 = time.perf_counter()
    while steps < steps_cap and time.perf_counter() - t0 < budget_s:
        one()
        steps += 1
    el = time.perf_counter() - t0
    o.set_pow_mode(0)
    return {"value": st.ny * st.nx * steps / el / 1e9, "unit": "Gcell-updates/s",
            "cores": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1)), "kind": "port",
            "steps": steps, "seconds": el}  # fmt: skip


def dambreak_spec() -> dict:
    z, depth = dambreak_inputs()
    return dict(scheme="hllc_fv", bed=z, dx=DX, depth=depth, manning=0.0, alpha=ALPHA, dt_max=DT_MAX)


def cpu_baseline(budget_s: float = 10.0) -> dict:
    """The CPU oracle (the reference's kernels restated in C, OpenMP over all host
    cores, libm powf as the reference's CPU build) on the full headline grid."""
    out = cpu_leg(dambreak_spec(), budget_s=budget_s, warmup=2)
    out["sample"] = (f"{out['steps']} HLLC steps (compute_dt + step) of the full {N}x{N} dam break after 2 untimed "
                     f"steps, C oracle (oracle/rbo.c) with OpenMP, {out['seconds']:.1f} s")
    return out


def run_reference(args) -> None:
    """The reference path's CPU implementation (the oracle port: its Warp CPU device
    cannot be installed here) on the headline configuration itself: W untimed warm-up
    steps, then K timed steps of the full 2048 x 2048 grid on all host cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    o = oracle_module()
    o.set_pow_mode(0)
    st, _ = oracle_state(dambreak_spec(), np.float32)
    for _ in range(args.warmup):
        o.hllc_step(st, o.hllc_compute_dt(st, ALPHA, DT_MAX))
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o.hllc_step(st, o.hllc_compute_dt(st, ALPHA, DT_MAX))
    el = time.perf_counter() - t0
    cells = N * N
    value = cells * args.steps / el / 1e9
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    line = {
        "impl": "reference", "metric": "Gcell-updates/s", "value": value, "unit": "Gcell-updates/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "grid": [N, N], "dx_m": DX, "alpha": ALPHA, "scheme": "hllc_fv",
                   "boundaries": "closed"},
        "cpu_baseline": {"value": value, "unit": "Gcell-updates/s", "cores": cores, "kind": "port",
                         "sample": f"each step one HLLC step (compute_dt + step) of the full {N}x{N} dam break, "
                                   f"after {args.warmup} untimed steps (the reference's Warp CPU device is not "
                                   "installable; C restatement of its kernels, OpenMP, libm powf)"},
        "e2e": {"value": value, "unit": "Gcell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }  # fmt: skip
    print(json.dumps(line))


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="rbsim", choices=["rbsim", "reference"])
    ap.add_argument("--workload", default="hllc_dambreak",
                    choices=["hllc_dambreak", "li_rain_512", "li_rain_2048", "hllc_lake_2048", "li_reach_8192",
                             "ensemble_256", "serve"],
                    help="hllc_dambreak is the headline; the others measure the remaining configurations")
    ap.add_argument("--arith", default="fast", choices=["exact", "fast"],
                    help="arithmetic of the step kernels for the headline (the other build is timed beside it)")
    ap.add_argument("--hllc-variant", type=int, default=None,
                    help="HLLC stage-kernel variant for the headline (rb_hllc_set_kernel_variant; default: the "
                         "library's)")
    ap.add_argument("--headline-only", action="store_true",
                    help="time the headline steps only (no e2e, other configurations, CPU or float64 legs)")
    ap.add_argument("--no-legs", action="store_true", help="skip the CPU and float64 legs of a --workload record")
    ap.add_argument("--rates", default="2,10,50", help="serve: arrival rates, requests/s")
    ap.add_argument("--requests", type=int, default=16, help="serve: requests per rate")
    args = ap.parse_args(argv)
    if args.workload != "hllc_dambreak" and args.impl == "rbsim":
        import bench_workloads

        out = bench_workloads.run(args)
        if int(os.environ.get("RANK", "0")) == 0:
            print(json.dumps(out))
        return 0
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        run_reference(args)
        return 0

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    import ctypes

    import rbsim
    from rbsim import _lib, arith, graphs, replicas
    from rbsim.device_clock import DeviceClock
    from rbsim.schemes import hllc

    L = _lib.lib()
    z, depth = dambreak_inputs()
    cells = N * N
    stream = torch.cuda.current_stream(dev)
    K = args.steps

    def timed_replay(sample_clocks: bool):
        """K device-resident steps, one CUDA graph, inputs resident, after W warm-up steps;
        then the same clocked steps launched one by one with events around each stage."""
        st = rbsim.State.from_bed(z, DX, depth=depth, manning=0.0, device=dev)
        hllc.arm_hllc(st)
        clk = DeviceClock(st, "hllc_fv", alpha=ALPHA, dt_max=DT_MAX, sync_times=[T_END], graph_steps=K)
        f = st.hllc_fields()
        ws = st.workspace.data_ptr()
        graph = graphs.capture(dev, lambda s: _lib.check(L.rb_hllc_enqueue_steps(ctypes.byref(f), K, 0, ws, s)))
        for _ in range(args.warmup):  # W untimed warm-up steps
            clk.set_target(T_END, 1)
            _lib.check(L.rb_hllc_enqueue_steps(ctypes.byref(f), 1, 0, ws, stream.cuda_stream))
        clk.set_target(T_END, K)
        barrier()
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local if sample_clocks else -1) as clocks:
            start.record(stream)
            graph.replay()
            stop.record(stream)
            barrier()
        ms = start.elapsed_time(stop)
        cs = clk.read()
        if cs.steps != args.warmup + K:
            raise RuntimeError(f"device clock took {cs.steps} steps, expected {args.warmup + K}")
        del graph
        ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(min(K, 50))]
        clk.set_target(T_END, len(ev))
        for e in ev:
            _lib.check(L.rb_clock_plan(ws, stream.cuda_stream))
            e[0].record(stream)
            _lib.check(L.rb_hllc_stage_clocked(ctypes.byref(f), 1, ws, stream.cuda_stream))
            e[1].record(stream)
            _lib.check(L.rb_hllc_stage_clocked(ctypes.byref(f), 2, ws, stream.cuda_stream))
            e[2].record(stream)
        torch.cuda.synchronize(dev)
        clk.read()
        clk.close()
        st.check_device_errors()
        return ms, clocks, [e[0].elapsed_time(e[1]) for e in ev], [e[1].elapsed_time(e[2]) for e in ev]

    # --- value: the selected arithmetic; then the other build, for comparison ---
    if args.hllc_variant is not None:
        _lib.check(L.rb_hllc_set_kernel_variant(args.hllc_variant))
    arith.set_arithmetic(args.arith)
    ms, clocks, stage1_ms, stage2_ms = timed_replay(True)
    # Whole job: the cells every replica stepped over the slowest replica's time.
    value, sec = replicas.whole_job_rate(cells * K / 1e9, ms / 1e3)
    ms = sec * 1e3
    other = "exact" if args.arith == "fast" else "fast"
    arith.set_arithmetic(other)
    ms_o, _, _, _ = timed_replay(False)
    value_o, sec_o = replicas.whole_job_rate(cells * K / 1e9, ms_o / 1e3)
    arith.set_arithmetic(args.arith)
    if args.headline_only:
        if rank == 0:
            print(json.dumps({"metric": "Gcell-updates/s", "value": value, "ms_per_step": ms / K, "build": args.arith,
                              "other_build": {"build": other, "value": value_o, "ms_per_step": sec_o * 1e3 / K}}))
        if world > 1:
            dist.destroy_process_group()
        return 0

    e2e = _e2e(args, dev, barrier, z, depth)

    # --- the other configurations' records: the LI roofline point and the largest
    # single-GPU configuration, each with its own roofline, CPU baseline and error ---
    import bench_workloads

    legs = world == 1
    sub = {"li_rain_2048": bench_workloads.li_rain_2048(args, legs=legs),
           "li_reach_8192": bench_workloads.li_reach_8192(args, legs=legs)}  # fmt: skip
    for rec in sub.values():  # whole job: every replica's cell-updates over the slowest replica's time
        roof = rec["roofline"]
        rec["value"], _ = replicas.whole_job_rate(roof["cell_updates"] / 1e9, roof["timed_s"])
        rec["n_gpus"] = world
    err64 = bench_workloads.f64_leg(dambreak_spec(), steps=12) if legs else None

    if rank == 0:
        pk = peaks()
        # roofline from the timed region itself: the step's algorithmic bytes over the
        # replayed step's event time (which also holds the one-thread plan kernel, so
        # this is a lower bound for the two stage kernels)
        achieved = BYTES_PER_CELL_STEP * cells / (ms / K / 1e3) / 1e9
        mean_kernel_ms = statistics.mean(a + b for a, b in zip(stage1_ms, stage2_ms, strict=True))
        line = {
            "metric": "Gcell-updates/s", "value": value, "unit": "Gcell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "grid": [N, N], "dx_m": DX, "alpha": ALPHA, "scheme": "hllc_fv",
                       "boundaries": "closed", "parallelism": f"replicas{world}", "build": BUILDS[args.arith],
                       "l2": "inputs larger than L2: 11 float32 fields of 16.8 MB (h, hu, hv double-buffered, "
                             "stage-1 state, z, n) = 185 MB touched per step vs 126 MB L2",
                       "step_loop": "device-resident clock (dt, fill_span, rain gating on the GPU), K steps "
                                     "replayed as one CUDA graph"},
            "gpu_launches": 3 * K,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                         "frac": achieved / pk["hbm_gbs"], "traffic": NCU_DRAM_BYTES_PER_STEP,
                         "traffic_note": "DRAM bytes read + written by stage 1 + stage 2 of one step, from one "
                                         "ncu capture of this workload; the algorithmic bytes per step are 134 MB",
                         "peak_source": pk["source"],
                         "timing": "CUDA events around the timed replay of K steps (stage 1 + stage 2 + the "
                                   "one-thread plan kernel per step): a lower bound for the stage pair",
                         "issue_bound": {"issue_slots_busy_stage1": NCU_ISSUE_ACTIVE[0],
                                         "issue_slots_busy_stage2": NCU_ISSUE_ACTIVE[1],
                                         "source": "the same ncu capture"},
                         "kernel": "hllc_stage_kernel stage 1 + stage 2 (one SSP-RK2 step)",
                         "bytes_per_cell_step": BYTES_PER_CELL_STEP,
                         "launched_one_by_one": {"stage_pair_ms_mean": mean_kernel_ms,
                                                 "stage1_ms_mean": statistics.mean(stage1_ms),
                                                 "stage2_ms_mean": statistics.mean(stage2_ms),
                                                 "note": f"{len(stage1_ms)} clocked steps launched one by one with "
                                                         "events around each stage (launch gaps included)"}},
            "clocks": clocks.summary(),
            "other_build": {"build": BUILDS[other], "value": value_o, "ms_per_step": sec_o * 1e3 / K},
            "e2e": e2e,
            "cpu_baseline": cpu_baseline() if legs else None,
            "err_vs_f64": err64,
            "workloads": sub,
        }  # fmt: skip
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


def _e2e(args, dev, barrier, z, depth) -> dict:
    """The headline metric end to end through the public API, from and to pinned host memory."""
    import torch

    import rbsim
    from rbsim import replicas
    from rbsim.device_clock import DeviceClock
    from rbsim.schemes import hllc

    K = args.steps
    cells = N * N
    # The job's inputs and result live in pinned host memory (staged before timing);
    # each timed run copies the bed and the initial depth in and the final depth out.
    z_host = torch.from_numpy(z).pin_memory()
    depth_host = torch.from_numpy(depth).pin_memory()
    h_host = torch.empty((N, N), dtype=torch.float32, pin_memory=True)

    def e2e_device_clock():
        st2 = rbsim.State.from_bed(z_host, DX, depth=depth_host, manning=0.0, device=dev)
        hllc.arm_hllc(st2)
        c2 = DeviceClock(st2, "hllc_fv", alpha=ALPHA, dt_max=DT_MAX, sync_times=[T_END], graph_steps=64)
        c2.run_until(T_END, max_steps=K)
        h_host.copy_(st2.h)
        c2.close()
        return h_host.numpy()

    def e2e_per_step_api():
        st3 = rbsim.State.from_bed(z_host, DX, depth=depth_host, manning=0.0, device=dev)
        hllc.arm_hllc(st3)
        for _ in range(K):
            hllc.step(st3, hllc.compute_dt(st3, alpha=ALPHA, dt_max=DT_MAX))
        h_host.copy_(st3.h)
        return h_host.numpy()

    e2e_device_clock()  # warms the allocator and the kernels outside the timing
    timings = {}
    for name, fn in (("device_clock", e2e_device_clock), ("per_step_api", e2e_per_step_api)):
        barrier()
        t0 = time.perf_counter()
        h_out = fn()
        barrier()
        timings[name], _ = replicas.whole_job_rate(cells * K / 1e9, time.perf_counter() - t0)
        assert np.isfinite(h_out).all()
    return {"value": timings["device_clock"], "unit": "Gcell-updates/s",
            "api": "State.from_bed + DeviceClock.run_until + a read of the final depth, from and to pinned host "
                   "memory", "h2d_bytes_per_step": 2 * 4 * cells / K, "d2h_bytes_per_step": 4 * cells / K,
            "per_step_api": {"value": timings["per_step_api"],
                             "api": "compute_dt + step per step (dt read back every step, as the reference's "
                                    "scheme API does)"}}  # fmt: skip


if __name__ == "__main__":
    sys.exit(main())
