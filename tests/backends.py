"""Two interchangeable backends for the physics gates: the CPU oracle and the CUDA path."""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np


class OracleBackend:
    name = "oracle"

    def __init__(self):
        import oracle

        self.o = oracle
        oracle.set_pow_mode(1)

    def make(self, bed, dx, depth=0.0, manning=0.035):
        return self.o.State.from_bed(bed, dx, depth=depth, manning=manning)

    def arm_hllc(self, st):
        st.arm_hllc()

    def set_hu(self, st, hu, hv):
        st.arm_hllc()
        st.hu[...] = hu
        st.hv[...] = hv

    def set_qx(self, st, qx):
        st.qx[...] = qx

    def arm_comp(self, st):
        st.arm_source_compensation()

    def set_infil(self, st, f):
        st.set_infiltration(f)

    def set_rain(self, st, f):
        st.set_rain_field(f)

    def set_bc(self, st, bc, curves=None):
        st.set_open_boundaries(bc, curves)

    def arm_channels(self, st, w, d, n=None):
        st.arm_channels(w, d, n)

    def reservoir(self, st, structure: dict):
        return self.o.ReservoirOperator(structure, st)

    def channel_n(self, st):
        return st.channels.n.copy()

    def compute_dt(self, st, scheme, alpha, dt_max):
        return self.o.SCHEMES[scheme][0](st, alpha, dt_max)

    def step(self, st, scheme, dt, rain=0.0, rain_scale=1.0, limit=True, t=0.0):
        if scheme == "hllc_fv":
            self.o.hllc_step(st, dt, rain=rain, rain_scale=rain_scale, t=t)
        else:
            self.o.li_step(st, dt, rain=rain, limit=limit, rain_scale=rain_scale, t=t)

    def h(self, st):
        return st.h.copy()

    def hu(self, st):
        return st.hu.copy()

    def hv(self, st):
        return st.hv.copy()

    def qx(self, st):
        return st.qx.copy()

    def qy(self, st):
        return st.qy.copy()

    def hcomp(self, st):
        return st.h_comp.copy()

    def velocities(self, st):
        return st.velocities()

    def loss_volume(self, st):
        return st.loss_volume()

    def ledger(self, st):
        led = self.o.MassLedger(st)

        class _L:
            def add_inflow(self, v):
                led.add_inflow(v)

            def add_rain_step(self, r, dt, n):
                led.add_rain_step(r, dt, n)

            def record(self, st_, t):
                return SimpleNamespace(**led.record(st_, t))

            @property
            def max_rel_error(self):
                return led.max_rel_error

            @property
            def v0(self):
                return led.v0

        return _L()

    def injector(self, inflows, st, compensated=True):
        infl = [self.o.Inflow(tuple(c), list(h)) for c, h in inflows]
        return self.o.InflowInjector(infl, st.ny, st.nx, st.dx, compensated=compensated)

    def n_cells(self, st):
        return st.ny * st.nx

    def cell_area(self, st):
        return st.dx * st.dx

    def fill_span(self, span, dt_raw):
        return self.o.fill_span(span, dt_raw)

    def arm_sediment(self, st, d50, porosity):
        st.arm_sediment(d50, porosity)

    def morphology(self, st, interval_s, dz_lo, dz_hi):
        """An object whose ``advance(t, dt_slow)`` applies one Exner activation."""
        o = self.o

        class _Morph:
            def advance(self, t, dt_slow):
                o.exner_activate(st, dz_lo, dz_hi)

        return _Morph()

    def z(self, st):
        return st.z.copy()

    def dz_cum(self, st):
        return st.sediment.dz_cum.copy()


class GpuBackend:
    name = "cuda"

    def __init__(self):
        import rbsim

        self.rb = rbsim

    def make(self, bed, dx, depth=0.0, manning=0.035):
        return self.rb.State.from_bed(bed, dx, depth=depth, manning=manning)

    def arm_hllc(self, st):
        st.arm_hllc_fields()

    def set_hu(self, st, hu, hv):
        st.arm_hllc_fields()
        st.hu = hu
        st.hv = hv

    def set_qx(self, st, qx):
        st.qx = qx

    def arm_comp(self, st):
        st.arm_source_compensation()

    def set_infil(self, st, f):
        st.set_infiltration(f)

    def set_rain(self, st, f):
        st.set_rain_field(f)

    def set_bc(self, st, bc, curves=None):
        st.set_open_boundaries(bc, curves)

    def arm_channels(self, st, w, d, n=None):
        from rbsim.channels import arm_channels

        arm_channels(st, w, d, n)

    def reservoir(self, st, structure: dict):
        from rbsim.config import Structure
        from rbsim.processes.reservoir import ReservoirOperator

        return ReservoirOperator(Structure(**structure), st)

    def channel_n(self, st):
        return st.channels.n.cpu().numpy()

    def compute_dt(self, st, scheme, alpha, dt_max):
        return self.rb.get_scheme(scheme).compute_dt(st, alpha=alpha, dt_max=dt_max)

    def step(self, st, scheme, dt, rain=0.0, rain_scale=1.0, limit=True, t=0.0):
        if scheme == "hllc_fv":
            self.rb.get_scheme(scheme).step(st, dt=dt, rain=rain, rain_scale=rain_scale, t=t)
        else:
            self.rb.get_scheme(scheme).step(st, dt=dt, rain=rain, limit=limit, rain_scale=rain_scale, t=t)

    def h(self, st):
        return st.h.cpu().numpy()

    def hu(self, st):
        return st.hu.cpu().numpy()

    def hv(self, st):
        return st.hv.cpu().numpy()

    def qx(self, st):
        return st.qx.cpu().numpy()

    def qy(self, st):
        return st.qy.cpu().numpy()

    def hcomp(self, st):
        return st.h_comp.cpu().numpy()

    def velocities(self, st):
        return st.velocities_numpy()

    def loss_volume(self, st):
        return st.loss_volume(st.grid.cell_area)

    def ledger(self, st):
        from rbsim.massbalance import MassLedger

        return MassLedger.from_state(st)

    def injector(self, inflows, st, compensated=True):
        from rbsim.processes.inflow import Inflow, InflowInjector

        infl = [Inflow(tuple(c), list(h)) for c, h in inflows]
        return InflowInjector(infl, st.grid, st.device, compensated=compensated)

    def n_cells(self, st):
        return st.grid.n_cells

    def cell_area(self, st):
        return st.grid.cell_area

    def fill_span(self, span, dt_raw):
        from rbsim.scheduler import fill_span

        return fill_span(span, dt_raw)

    def arm_sediment(self, st, d50, porosity):
        from rbsim.sediment import arm_sediment

        arm_sediment(st, d50, porosity)

    def morphology(self, st, interval_s, dz_lo, dz_hi):
        from rbsim.processes.morphology import MorphologyProcess

        return MorphologyProcess(st, interval_s, dz_lo=dz_lo, dz_hi=dz_hi)

    def z(self, st):
        return st.z.cpu().numpy()

    def dz_cum(self, st):
        return st.sediment.dz_cum.cpu().numpy()


def flat(n, depth, be, dx=100.0):
    return be.make(np.zeros((n, n), np.float32), dx, depth=depth, manning=0.03)


def as_f64(a):
    return np.asarray(a, dtype=np.float64)
