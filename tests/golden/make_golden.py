"""Generate the committed golden fixtures by running the reference's own kernels.

Usage (in a checkout that has the reference tree; nothing else reads it):

    python tests/golden/make_golden.py --reference /path/to/river-basin-sim

The reference solver is NVIDIA Warp code. Warp is not installable here, so
``fake_warp.py`` is registered as ``warp`` and the reference modules
(``solver/core/*``, ``solver/processes/*``) are imported unmodified from the
reference tree; their ``@wp.kernel`` bodies then execute one thread index at a
time with float32 scalars (see ``fake_warp.py`` for the arithmetic model). Each
case of ``cases.py`` is stepped through the reference's own ``compute_dt`` /
``step`` / ``InflowInjector.apply`` / ``MorphologyProcess.advance`` and the end
state is written to ``<case>.npz`` beside this script.
"""

from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


class ReferenceAPI:
    def __init__(self):
        from solver.core import hllc, local_inertial
        from solver.core.channels import arm_channels
        from solver.core.sediment import arm_sediment
        from solver.core.state import State
        from solver.io.config import Inflow
        from solver.processes.inflow import InflowInjector
        from solver.io.config import Structure
        from solver.processes.morphology import MorphologyProcess
        from solver.processes.reservoir import ReservoirOperator

        self.State = State
        self.schemes = {"local_inertial": local_inertial, "hllc_fv": hllc}
        self.hllc = hllc
        self.arm_sediment = arm_sediment
        self.arm_channels = arm_channels
        self.Inflow = Inflow
        self.InflowInjector = InflowInjector
        self.MorphologyProcess = MorphologyProcess
        self.Structure = Structure
        self.ReservoirOperator = ReservoirOperator
        self.case = None

    def make_state(self, case):
        import warp as wp

        self.case = case
        st = self.State.from_bed(case["bed"], dx=case["dx"], depth=case["depth"], manning=case["manning"],
                                 device="cpu")  # fmt: skip
        if case["scheme"] == "hllc_fv":
            self.hllc.arm_hllc(st)
            if "hu0" in case:
                st.hu.assign(case["hu0"])
                st.hv.assign(case["hv0"])
        if "qx0" in case:
            st.qx = wp.array(case["qx0"], dtype=wp.float32, device="cpu")
        if "infil" in case:
            st.set_infiltration(case["infil"])
        if "rain_field" in case:
            st.set_rain_field(case["rain_field"])
        if case.get("compensated"):
            st.arm_source_compensation()
        if "boundaries" in case:
            st.set_open_boundaries(case["boundaries"], case.get("stage_curves"))
        if case.get("sediment"):
            self.arm_sediment(st, case["sediment"]["d50"], case["sediment"]["porosity"])
        if case.get("channels"):
            ch = case["channels"]
            self.arm_channels(st, ch["width"], ch["depth"], ch.get("manning"))
        return st

    def compute_dt(self, st, alpha, dt_max):
        return self.schemes[self.case["scheme"]].compute_dt(st, alpha=alpha, dt_max=dt_max)

    def step(self, st, dt, rain, rain_scale, t):
        self.schemes[self.case["scheme"]].step(st, dt=dt, rain=rain, rain_scale=rain_scale, t=t)

    def injector(self, case, st):
        from solver.core.grid import Grid

        infl = [self.Inflow(cell=tuple(c), hydrograph=list(h)) for c, h in case["inflows"]]
        ny, nx = case["bed"].shape
        return self.InflowInjector(infl, Grid(ny=ny, nx=nx, dx=float(case["dx"])), "cpu")

    def morphology(self, case, st):
        sed = case["sediment"]
        return self.MorphologyProcess(st, 1.0e9, dz_lo=sed["dz_lo"], dz_hi=sed["dz_hi"])

    def reservoir(self, case, st):
        return self.ReservoirOperator(self.Structure(**case["reservoir"]["structure"]), st)

    def outputs(self, st, case):
        out = {"h": st.h.numpy().copy()}
        if case["scheme"] == "hllc_fv":
            out["hu"] = st.hu.numpy().copy()
            out["hv"] = st.hv.numpy().copy()
        else:
            out["qx"] = st.qx.numpy().copy()
            out["qy"] = st.qy.numpy().copy()
        if st.h_comp is not None:
            out["h_comp"] = st.h_comp.numpy().copy()
        if st.loss_cum is not None:
            out["loss_cum"] = st.loss_cum.numpy().copy()
        if st.sediment is not None:
            sed = st.sediment
            for k in ("qs_int_x", "qs_comp_x", "qs_int_y", "qs_comp_y", "dz_cum", "dz_unapplied"):
                out[k] = getattr(sed, k).numpy().copy()
            out["z"] = st.z.numpy().copy()
        if st.channels is not None:
            for k in ("qx_ch", "qx_fp", "qy_ch", "qy_fp"):
                out[k] = getattr(st.channels, k).numpy().copy()
        return out


SCHEDULER_CASES = {
    # name: (end_time, output_every, events, [(process name, interval)], dt recipe)
    "plain": (3600.0, 600.0, [], [], ("const", 7.3)),
    "rain_and_knots": (7200.0, 900.0, [1800.0, 2.5, 3333.3], [], ("wave", 11.0)),
    "slow_processes": (5400.0, 1000.0, [1234.5], [("reservoir", 900.0), ("morphology", 600.0)], ("wave", 37.0)),
    "coarse_dt": (100.0, 30.0, [10.0], [("morphology", 25.0)], ("const", 1000.0)),
    "near_integer": (10.0, 1.0, [], [], ("const", 0.1)),
}


def _dt_fn(recipe):
    import math

    kind, base = recipe
    k = [0]

    def fn():
        k[0] += 1
        if kind == "const":
            return base
        return base * (1.0 + 0.35 * math.sin(0.37 * k[0]))

    return fn


def make_scheduler_fixture(out_path):
    """Record the reference scheduler's ticks for stub dt sequences (solver/scheduler.py)."""
    import json

    from solver.scheduler import MultiRateScheduler, SlowProcess

    out = {}
    for name, (end, every, events, procs, recipe) in SCHEDULER_CASES.items():
        sp = [SlowProcess(name=n, interval=iv, advance=lambda t, e: None) for n, iv in procs]
        sched = MultiRateScheduler(end_time=end, output_every=every, events=events, processes=sp)
        ticks = [[t.index, t.t0, t.dt, t.t1, t.is_output, [[p.name, el] for p, el in t.due]]
                 for t in sched.ticks(_dt_fn(recipe))]
        out[name] = {"n_frames": sched.n_frames, "sync": sched.sync_times, "ticks": ticks}
    with open(out_path, "w") as f:
        json.dump(out, f)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="root of the reference source tree")
    ap.add_argument("cases", nargs="*")
    args = ap.parse_args(argv)

    sys.path.insert(0, HERE)
    import fake_warp

    fake_warp.install()
    sys.path.insert(0, os.path.abspath(args.reference))
    from cases import CASES, COMBINED_CASES, run_case

    make_scheduler_fixture(os.path.join(HERE, "scheduler_ticks.json"))
    api = ReferenceAPI()
    every = {**CASES, **COMBINED_CASES}
    names = args.cases or list(every)
    for name in names:
        t0 = time.time()
        out = run_case(every[name](), api)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(f"{name}: {time.time() - t0:.1f}s  keys={sorted(out)}")


if __name__ == "__main__":
    main()
