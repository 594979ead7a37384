"""Adapter from the shared case recipe (tests/golden/cases.py) to the CUDA path.

Everything goes through the public package (``rbsim``): ``State``, the scheme
modules returned by ``get_scheme``, ``InflowInjector`` and ``MorphologyProcess``.
"""

from __future__ import annotations

import numpy as np

import rbsim
from rbsim.channels import arm_channels
from rbsim.grid import Grid
from rbsim.processes.inflow import Inflow, InflowInjector
from rbsim.processes.morphology import MorphologyProcess
from rbsim.schemes import hllc
from rbsim.sediment import arm_sediment


class GpuAPI:
    def __init__(self):
        self.case = None

    def make_state(self, case):
        self.case = case
        st = rbsim.State.from_bed(case["bed"], case["dx"], depth=case["depth"], manning=case["manning"])
        if case["scheme"] == "hllc_fv":
            hllc.arm_hllc(st)
            if "hu0" in case:
                st.hu = case["hu0"]
                st.hv = case["hv0"]
        if "qx0" in case:
            st.qx = case["qx0"]
        if "infil" in case:
            st.set_infiltration(case["infil"])
        if "rain_field" in case:
            st.set_rain_field(case["rain_field"])
        if case.get("compensated"):
            st.arm_source_compensation()
        if "boundaries" in case:
            st.set_open_boundaries(case["boundaries"], case.get("stage_curves"))
        if case.get("sediment"):
            arm_sediment(st, case["sediment"]["d50"], case["sediment"]["porosity"])
        if case.get("channels"):
            ch = case["channels"]
            arm_channels(st, ch["width"], ch["depth"], ch.get("manning"))
        return st

    def compute_dt(self, st, alpha, dt_max):
        return rbsim.get_scheme(self.case["scheme"]).compute_dt(st, alpha=alpha, dt_max=dt_max)

    def step(self, st, dt, rain, rain_scale, t):
        rbsim.get_scheme(self.case["scheme"]).step(st, dt=dt, rain=rain, rain_scale=rain_scale, t=t)

    def injector(self, case, st):
        infl = [Inflow(tuple(c), list(h)) for c, h in case["inflows"]]
        return InflowInjector(infl, Grid(st.grid.ny, st.grid.nx, st.grid.dx), st.device)

    def morphology(self, case, st):
        sed = case["sediment"]
        return MorphologyProcess(st, 1.0e9, dz_lo=sed["dz_lo"], dz_hi=sed["dz_hi"])

    def reservoir(self, case, st):
        from rbsim.config import Structure
        from rbsim.processes.reservoir import ReservoirOperator

        return ReservoirOperator(Structure(**case["reservoir"]["structure"]), st)

    def outputs(self, st, case):
        out = {"h": st.h.cpu().numpy()}
        if case["scheme"] == "hllc_fv":
            out["hu"], out["hv"] = st.hu.cpu().numpy(), st.hv.cpu().numpy()
        else:
            out["qx"], out["qy"] = st.qx.cpu().numpy(), st.qy.cpu().numpy()
        if st.h_comp is not None:
            out["h_comp"] = st.h_comp.cpu().numpy()
        if st.loss_cum is not None:
            out["loss_total"] = np.float64(st.loss_cum.total())
        if st.sediment is not None:
            sed = st.sediment
            for k in ("qs_int_x", "qs_comp_x", "qs_int_y", "qs_comp_y", "dz_cum", "dz_unapplied"):
                out[k] = getattr(sed, k).cpu().numpy()
            out["z"] = st.z.cpu().numpy()
        if st.channels is not None:
            for k in ("qx_ch", "qx_fp", "qy_ch", "qy_fp"):
                out[k] = getattr(st.channels, k).cpu().numpy()
        st.check_device_errors()
        return out
