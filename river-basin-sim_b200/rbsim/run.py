"""Run a scenario on the B200 and stream results to the Zarr store (solver/run.py:140-584).

Same arming order and hot-loop semantics as the reference ``run_simulation``:
barriers raised into the bed -> fields -> sub-grid channels -> morphology (z0
captured after the bed is final, structure cells frozen) -> infiltration -> rain
field -> areal-source compensation -> inflow injector -> boundaries -> reservoir
operators -> ledgers -> writer + frame 0 -> the scheduler's ticks: inject, step,
bank rain, advance due slow processes (reservoirs before morphology), record +
write at output ticks.

Two ways through the ticks, with identical results:

* the **device clock** (default): the scheduler's sync times, the hydrograph
  knots and the stage curves are uploaded once and the GPU plans and takes every
  step between host events (outputs, slow-process activations, the end) in
  CUDA-graph replays; the host wakes only for those.
* the **host loop** (``use_device_clock=False``): one ``compute_dt`` + ``step`` per
  tick exactly as the reference's run loop.

    python -m rbsim.run --config scenario.toml --out results.zarr [--status status.json]
        [--frames-dir frames] [--no-frames] [--host-loop]
"""

from __future__ import annotations

import argparse
import sys
import time
from pathlib import Path

import numpy as np
import torch

from .config import Scenario, load_config
from .grid import H_DRY
from .io.status import StatusWriter
from .io.zarr_writer import AsyncFrameWriter, ZarrWriter
from .massbalance import MassLedger, SedimentLedger
from .processes.inflow import InflowInjector
from .processes.morphology import MorphologyProcess, bed_change_bounds
from .processes.reservoir import apply_barriers, build_operators
from .scheduler import EPS_T, MultiRateScheduler
from .schemes import get_scheme, hllc
from .sediment import arm_sediment
from .state import State


def _cell_velocities(st: State):
    """state.py:232-256 on the device: (u, v) cell-centred, 0 where h < H_DRY."""
    h = st.h
    wet = h >= H_DRY
    if st.hu is not None:
        qx_c, qy_c = st.hu, st.hv
    else:
        qx_c = 0.5 * (st.qx[:, :-1] + st.qx[:, 1:])
        qy_c = 0.5 * (st.qy[:-1, :] + st.qy[1:, :])
    zero = torch.zeros_like(h)
    return torch.where(wet, qx_c / h, zero), torch.where(wet, qy_c / h, zero)


def run_simulation(scenario: Scenario, bed=None, out_path="results.zarr", *, device="cuda", verbose: bool = True,
                   status: StatusWriter | None = None, use_device_clock: bool = True,
                   graph_steps: int = 32) -> MassLedger:  # fmt: skip
    sc = scenario
    bed = sc.bed if bed is None else bed
    if bed is None:
        raise ValueError("no bed: pass an array or set [grid] dem")
    if sc.dx is None:
        raise ValueError("scenario.dx is unresolved")
    scheme = get_scheme(sc.scheme)
    bed = apply_barriers(np.asarray(bed, np.float32), sc.structures)  # run.py:199
    st = State.from_bed(bed, sc.dx, depth=sc.initial_depth, manning=sc.manning, device=device)
    grid = st.grid
    if sc.scheme == "hllc_fv":
        hllc.arm_hllc(st)

    channels = None
    if sc.has_channels:  # run.py:204-228
        from .channels import arm_channels

        shape = grid.shape
        channels = arm_channels(st, np.broadcast_to(np.asarray(sc.channel_width, np.float32), shape),
                                np.broadcast_to(np.asarray(sc.channel_depth, np.float32), shape),
                                None if sc.channel_manning is None
                                else np.broadcast_to(np.asarray(sc.channel_manning, np.float32), shape))  # fmt: skip
        if verbose:
            print(f"  channels      : {channels.summary()}")

    morphology = None
    if sc.has_sediment:
        arm_sediment(st, sc.sediment_d50, sc.sediment_porosity)
        frozen = [cell for s in sc.structures for cell in s.cells]  # run.py:252-258: dams do not scour
        dz_lo, dz_hi = bed_change_bounds(grid.shape, alluvium_thickness=sc.alluvium_thickness, frozen_cells=frozen)
        morphology = MorphologyProcess(st, sc.sediment_interval_s, dz_lo=dz_lo, dz_hi=dz_hi)
        if verbose:
            print(f"  morphology    : {morphology.summary()}")

    infil = np.broadcast_to(np.asarray(sc.infiltration_mm_hr, np.float32), grid.shape)
    infil_m_s = infil / 1000.0 / 3600.0
    if not np.isscalar(sc.infiltration_mm_hr) or float(infil_m_s.max()) > 0.0:
        st.set_infiltration(infil_m_s)
    rain_is_field = sc.rain_type == "field"
    rain_field_sum = 0.0
    if rain_is_field:
        rf = (np.asarray(sc.rain_field, np.float32) / 1000.0 / 3600.0).astype(np.float32)
        st.set_rain_field(rf)
        rain_field_sum = float(rf.astype(np.float64).sum())
    if rain_is_field or (sc.rain_m_s > 0.0 and sc.rain_duration > 0.0):
        st.arm_source_compensation()
    injector = InflowInjector(sc.inflows, grid, st.device) if sc.inflows else None
    st.set_open_boundaries(sc.boundaries, sc.stage_curves)
    reservoirs = build_operators(sc.structures, st)  # after the State: they arm the loss ledger

    ledger = MassLedger.from_state(st)
    sed_ledger = SedimentLedger.from_state(st) if morphology is not None else None
    n_frames = int(round(sc.end_time / sc.output_every)) + 1
    attrs = {
        "scheme": sc.scheme, "dx": grid.dx, "coarsen": 1,
        "units": {"depth": "m", "u": "m/s", "v": "m/s", "time": "s", "bed": "m"},
        "scenario": sc.name, "rain_type": sc.rain_type, "rain_mm_hr": sc.rain_mm_hr,
        "rain_duration_s": sc.rain_duration, "end_time_s": sc.end_time, "output_every_s": sc.output_every,
        "datum_shift_m": 0.0, "solver": "rbsim (B200 CUDA)",
    }  # fmt: skip
    if morphology is not None:
        attrs["sediment"] = {"law": "mpm", **morphology.as_attrs()}
    if channels is not None:
        attrs["channels"] = channels.as_attrs()
    writer = ZarrWriter(out_path, grid, n_frames, attrs, bed_change=morphology is not None)
    writer.write_bed(np.asarray(bed, np.float32))
    if channels is not None:  # run.py:331-335
        writer.write_static("channel_width", channels.w.cpu().numpy())
        writer.write_static("channel_depth", channels.d.cpu().numpy())
    frames = AsyncFrameWriter(writer, st.device)

    def emit(t_out: float) -> None:
        u, v = _cell_velocities(st)
        frames.submit(t_out, st.h, u, v, st.sediment.dz_cum if morphology is not None else None)

    emit(0.0)
    inflow_events = injector.breakpoints() if injector else []
    sched = MultiRateScheduler(
        end_time=sc.end_time, output_every=sc.output_every,
        events=[sc.rain_duration, *inflow_events, *sc.stage_events],
        processes=[*(r.as_slow_process() for r in reservoirs),
                   *([morphology.as_slow_process()] if morphology is not None else [])],
    )  # fmt: skip

    def on_output(t1: float) -> None:
        rec = ledger.record(st, t1)
        emit(t1)
        h_max = float(st.h.max().item())
        line = f"  t={t1:8.1f}s  h_max={h_max:6.3f}m  mass_rel_err={rec.rel_error:.2e}"
        if sed_ledger is not None:
            line += f"  bed_moved={sed_ledger.record(st, t1).gross_volume:9.1f}m3"
        if verbose:
            print(line)
        if status is not None:
            status.write("running", sim_time=t1,
                         message=f"t={t1:.0f}s  h_max={h_max:.3f}m  mass_rel_err={rec.rel_error:.1e}")  # fmt: skip

    if use_device_clock:
        from .device_clock import DeviceClock

        clock = DeviceClock(st, sc.scheme, alpha=sc.alpha, dt_max=sc.dt_max, sync_times=sched.sync_times,
                            rain_rate=0.0 if rain_is_field else sc.rain_m_s, rain_until=sc.rain_duration,
                            graph_steps=graph_steps, injector=injector)  # fmt: skip
        procs = [p for p in sched.processes]
        pending = {p.name: list(p.activations(sc.end_time)) for p in procs}
        last_ran = {p.name: 0.0 for p in procs}
        outputs = list(sched.output_times)
        targets = sorted({*outputs, *[t for ts in pending.values() for t in ts], sc.end_time})
        banked_rain = banked_inflow = 0.0
        next_output = sc.output_every
        for target in targets:
            if target <= clock.t + EPS_T:
                continue
            clock.run_until(target)
            t1 = clock.t
            ledger.add_inflow(clock.inflow_volume - banked_inflow)
            ledger.add_inflow(clock.rain_volume - banked_rain)
            banked_rain, banked_inflow = clock.rain_volume, clock.inflow_volume
            any_fired = False
            for p in procs:  # scheduler.py:234-242, on the step that landed here
                times, fired = pending[p.name], False
                while times and t1 >= times[0] - EPS_T:
                    times.pop(0)
                    fired = True
                if fired:
                    p.advance(t1, t1 - last_ran[p.name])
                    last_ran[p.name] = t1
                    any_fired = True
            if any_fired and reservoirs:  # a release moved water: the next dt reads the new state
                clock.reseed()
            if t1 >= next_output - EPS_T and next_output <= sc.end_time + EPS_T:
                next_output += sc.output_every
                on_output(t1)
        clock.close()
    else:
        for tick in sched.ticks(lambda: scheme.compute_dt(st, alpha=sc.alpha, dt_max=sc.dt_max)):
            t, dt = tick.t0, tick.dt
            if injector is not None:
                ledger.add_inflow(injector.apply(st, t, dt))
            raining = t < sc.rain_duration - EPS_T
            if rain_is_field:
                scheme.step(st, dt=dt, rain_scale=(1.0 if raining else 0.0), t=t)
                if raining:
                    ledger.add_inflow(rain_field_sum * dt * grid.cell_area)
            else:
                rain = sc.rain_m_s if raining else 0.0
                scheme.step(st, dt=dt, rain=rain, t=t)
                if rain > 0.0:
                    ledger.add_rain_step(rain, dt, grid.n_cells)
            for proc, elapsed in tick.due:
                proc.advance(tick.t1, elapsed)
            if tick.is_output:
                on_output(tick.t1)
    st.check_device_errors()
    frames.close()
    final = dict(ledger.as_attrs())
    if morphology is not None:
        final["morphology"] = morphology.series
        final.update(sed_ledger.as_attrs())
    if reservoirs:
        final["reservoir_releases"] = {r.structure.name: r.series for r in reservoirs}
    writer.finalize(final)
    if verbose and ledger.max_rel_error >= 1e-6:
        print(f"  warning: mass balance {ledger.max_rel_error:.2e} exceeds the 1e-6 gate")
    return ledger


def main(argv=None) -> int:
    """The run-loop CLI (solver/run.py:486-580): a scenario in, a result store, the
    viewer's frames and ``status.json`` out."""
    ap = argparse.ArgumentParser(prog="python -m rbsim.run")
    ap.add_argument("--config", required=True, help="scenario TOML")
    ap.add_argument("--out", default=None, help="result store; default <config name>.zarr")
    ap.add_argument("--status", default=None, help="status.json path; default <out-dir>/status.json")
    ap.add_argument("--frames-dir", default=None, help="viewer frames; default <out-dir>/frames")
    ap.add_argument("--no-frames", action="store_true", help="skip the viewer frame export")
    ap.add_argument("--host-loop", action="store_true", help="step through compute_dt/step on the host")
    args = ap.parse_args(argv)
    out = Path(args.out or Path(args.config).with_suffix(".zarr").name)
    out.parent.mkdir(parents=True, exist_ok=True)
    # The status channel opens before anything that can fail, the config included, so a
    # viewer polling it sees state "error" rather than a file that never appears. Its
    # end time is set once the scenario is known.
    status = StatusWriter(args.status or out.parent / "status.json", 1.0)
    try:
        status.write("starting", message="reading the scenario")
        sc = load_config(args.config)
        status.end_time = float(sc.end_time)
        status.write("starting", message=sc.name)
        t0 = time.time()
        ledger = run_simulation(sc, None, str(out), status=status, use_device_clock=not args.host_loop)
        if not args.no_frames:
            from .io.viewer_export import export_frames

            status.write("writing", sim_time=sc.end_time, message="exporting viewer frames")
            export_frames(out, args.frames_dir or out.parent / "frames")
        status.write("done", sim_time=sc.end_time,
                     message=f"mass_max_rel_err={ledger.max_rel_error:.2e}, wall {time.time() - t0:.1f}s")  # fmt: skip
    except Exception as e:
        status.write("error", message=f"{type(e).__name__}: {e}")
        raise
    return 0


if __name__ == "__main__":
    sys.exit(main())
