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
        from solver.core.sediment import arm_sediment
        from solver.core.state import State
        from solver.io.config import Inflow
        from solver.processes.inflow import InflowInjector
        from solver.processes.morphology import MorphologyProcess

        self.State = State
        self.schemes = {"local_inertial": local_inertial, "hllc_fv": hllc}
        self.hllc = hllc
        self.arm_sediment = arm_sediment
        self.Inflow = Inflow
        self.InflowInjector = InflowInjector
        self.MorphologyProcess = MorphologyProcess
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
        return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="root of the reference source tree")
    ap.add_argument("cases", nargs="*")
    args = ap.parse_args(argv)

    sys.path.insert(0, HERE)
    import fake_warp

    fake_warp.install()
    sys.path.insert(0, os.path.abspath(args.reference))
    from cases import CASES, run_case

    api = ReferenceAPI()
    names = args.cases or list(CASES)
    for name in names:
        t0 = time.time()
        out = run_case(CASES[name](), api)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(f"{name}: {time.time() - t0:.1f}s  keys={sorted(out)}")


if __name__ == "__main__":
    main()
