"""A request loop that serves scenario solves with continuous batching.

Requests (scheme, grid side, horizon, seeded synthetic terrain, optional Exner
morphology) arrive over wall-clock time. The server admits them in arrival order
while the HBM they need fits the budget, keeps every admitted solve resident, and
steps all of them together as one ``Ensemble`` (one persistent kernel per scheme
over the members' tiles, the single-domain kernels for members large enough to fill
the GPU alone; each member on its own device clock). Between graph
replays it retires finished solves (their results at once; a finished member stays
in the batch, idle, until the next rebuild -- an admission, or finished members
holding most of the batch's cells -- frees its memory), runs due slow processes
(Exner activations) for the members that reached them, streams output frames, and
admits whatever arrived meanwhile -- so new work joins the batch while older work
is still on the GPU. Each result is bit-identical to solving that request alone
(``solve_alone``), frames included.

Frames. With ``out_dir`` set, every request with ``output_every > 0`` gets its own
result store (``req_<rid>.zarr``, the layout of ``rbsim.io.zarr_writer``, as the
reference's run loop writes one per run, solver/run.py:329-429): frame 0 at
admission, then one frame at every multiple of ``output_every`` and at the horizon
(each member's clock lands on those times exactly). A frame's fields are copied
device-to-host on a side stream into pinned buffers and written by one writer
thread (``FrameStream``), so the batch keeps stepping while frames travel; a
bounded queue holds at most ``max_pending_frames`` frames in flight.

``serial_baseline`` solves the same requests one after another, each alone, in
arrival order: the plain loop the batched server is measured against.
"""

from __future__ import annotations

import math
import queue
import threading
import time
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np
import torch

from .ensemble import Ensemble
from .grid import H_DRY
from .io.zarr_writer import ZarrWriter
from .processes.morphology import MorphologyProcess
from .scheduler import EPS_T
from .sediment import arm_sediment
from .state import State

ALPHA = {"local_inertial": 0.7, "hllc_fv": 0.45}


@dataclass
class Request:
    rid: int
    arrival: float  # seconds after the stream starts
    scheme: str  # "local_inertial" | "hllc_fv"
    side: int  # grid side, cells
    horizon: float  # simulated seconds
    seed: int
    exner: bool = False
    dx: float = 10.0
    rain_mm_hr: float = 30.0
    morph_interval: float = 300.0
    output_every: float = 0.0  # simulated seconds between frames; 0: no frames


@dataclass
class Result:
    rid: int
    arrival: float
    admitted: float
    finished: float
    steps: int
    t: float
    depth: np.ndarray | None = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def request_bytes(req: Request) -> int:
    """Device bytes a request holds while resident (fields, workspace, morphology)."""
    n = req.side * req.side
    if req.scheme == "hllc_fv":
        per = 4 * (6 + 2 + 3)  # h/hu/hv double-buffered, z, n, stage-1 state
    else:
        per = 4 * (6 + 2 + 1)  # h/qx/qy double-buffered, z, n, rain residue
        if req.exner:
            per += 4 + 4 + 8 + 8 + 16  # d50, z0, dz_cum, dz_unapplied, four transport accumulators
    return per * n + (1 << 20)


def output_times(req: Request) -> list[float]:
    """Frame times after t = 0: multiples of ``output_every`` up to the horizon, and the horizon."""
    if req.output_every <= 0.0:
        return []
    out, k = [], 1
    while k * req.output_every < req.horizon - EPS_T:
        out.append(k * req.output_every)
        k += 1
    return out + [req.horizon]


def _cell_velocities(st: State):
    """Cell-centred (u, v) on the device, 0 where h < H_DRY (state.py:232-256)."""
    h = st.h
    if st.hu is not None:
        qx, qy = st.hu, st.hv
    else:
        qx = 0.5 * (st.qx[:, :-1] + st.qx[:, 1:])
        qy = 0.5 * (st.qy[:-1, :] + st.qy[1:, :])
    wet = h >= H_DRY
    zero = torch.zeros_like(h)
    return torch.where(wet, qx / h, zero), torch.where(wet, qy / h, zero)


class FrameStream:
    """Frames of every served request to that request's store, off the compute path.

    ``submit`` orders a frame's device-to-host copies on a side stream after the
    compute stream's work so far, into pinned buffers, and queues the write; one
    thread waits for each copy to land and appends it to its store. ``finish``
    queues a store's finalisation behind its frames. The queue is bounded, so at
    most ``max_pending`` frames' buffers are in flight.
    """

    def __init__(self, device, max_pending: int = 8):
        self.device = device
        self._side = torch.cuda.Stream(device)
        self._jobs: queue.Queue = queue.Queue(maxsize=max(1, int(max_pending)))
        self._error: BaseException | None = None
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._thread.start()
        self.frames = 0

    def submit(self, writer: ZarrWriter, t: float, fields: list) -> None:
        if self._error is not None:
            raise self._error
        ready = torch.cuda.Event()
        ready.record(torch.cuda.current_stream(self.device))
        self._side.wait_event(ready)
        with torch.cuda.stream(self._side):
            bufs = []
            for f in fields:
                b = torch.empty(f.shape, dtype=torch.float32, pin_memory=True)
                b.copy_(f, non_blocking=True)
                f.record_stream(self._side)
                bufs.append(b)
            done = torch.cuda.Event()
            done.record(self._side)
        self._jobs.put(("frame", writer, float(t), done, bufs))
        self.frames += 1

    def finish(self, writer: ZarrWriter, attrs: dict) -> None:
        self._jobs.put(("finish", writer, attrs))

    def _run(self) -> None:
        while True:
            job = self._jobs.get()
            if job is None:
                return
            try:
                if job[0] == "frame":
                    _, writer, t, done, bufs = job
                    done.synchronize()
                    arrs = [b.numpy() for b in bufs]
                    writer.append(t, arrs[0], arrs[1], arrs[2], arrs[3] if len(arrs) > 3 else None)
                else:
                    job[1].finalize(job[2])
            except BaseException as e:  # surfaced on the next submit / close
                self._error = e

    def close(self) -> None:
        self._jobs.put(None)
        self._thread.join()
        if self._error is not None:
            raise self._error


def build_state(req: Request, device) -> tuple[State, MorphologyProcess | None]:
    """Seeded synthetic terrain: a sloping plane plus Gaussian bumps, rain-on-grid."""
    rng = np.random.default_rng(req.seed)
    n = req.side
    yy, xx = np.mgrid[0:n, 0:n].astype(np.float32)
    z = 1e-3 * xx * req.dx
    for _ in range(6):
        a, s = rng.uniform(0.5, 3.0), rng.uniform(3.0, 0.2 * n)
        cy, cx = rng.uniform(0, n), rng.uniform(0, n)
        z += a * np.exp(-((yy - cy) ** 2 + (xx - cx) ** 2) / (2 * s * s))
    manning = float(rng.uniform(0.02, 0.06))
    depth = 0.05 if req.scheme == "local_inertial" else np.where(xx < n / 2, 1.0, 0.2).astype(np.float32)
    st = State.from_bed(z.astype(np.float32), req.dx, depth=depth, manning=manning, device=device)
    morph = None
    if req.scheme == "hllc_fv":
        st.arm_hllc_fields()
    else:
        st.arm_source_compensation()
        st.set_open_boundaries({"east": "open"})
        if req.exner:
            arm_sediment(st, 0.002, 0.4)
            morph = MorphologyProcess(st, req.morph_interval)
    return st, morph


@dataclass
class _Member:
    req: Request
    st: State
    morph: MorphologyProcess | None
    admitted: float
    nbytes: int
    next_act: float = math.inf  # next Exner activation (simulated s)
    last_act: float = 0.0
    t: float = 0.0  # simulated time reached
    steps: int = 0  # steps taken
    base_steps: int = 0  # steps taken before the current ensemble was built
    writer: ZarrWriter | None = None  # the request's result store, when frames are streamed
    outputs: list[float] = field(default_factory=list)  # frame times still to come
    done: bool = False  # reached its horizon; leaves the batch at the next rebuild

    @property
    def target(self) -> float:
        return min(self.next_act, self.outputs[0] if self.outputs else math.inf, self.req.horizon)

    def sync_times(self) -> list[float]:
        acts = []
        if self.morph is not None:
            k = 1
            while k * self.req.morph_interval <= self.req.horizon + EPS_T:
                acts.append(k * self.req.morph_interval)
                k += 1
        return sorted({*acts, *output_times(self.req), self.req.horizon})

    def frame_fields(self) -> list:
        """The frame's fields as fresh device tensors: the depth is snapshotted on the
        compute stream, because the steps that follow write its buffer again while the
        side stream may still be copying."""
        u, v = _cell_velocities(self.st)
        extra = [self.st.sediment.dz_cum.float()] if self.morph is not None else []
        return [self.st.h.clone(), u, v, *extra]


def _build_ensemble(members: list[_Member], graph_steps: int) -> Ensemble:
    """An ensemble over the current members, each clock continuing from where it stopped."""
    reqs = [m.req for m in members]
    for m in members:
        m.base_steps = m.steps
    ens = Ensemble(
        [m.st for m in members], [r.scheme for r in reqs], alpha=[ALPHA[r.scheme] for r in reqs], dt_max=30.0,
        sync_times=[m.sync_times() for m in members], rain_rate=[r.rain_mm_hr / 3.6e6 for r in reqs],
        rain_until=[r.horizon for r in reqs], graph_steps=graph_steps, t0=[m.t for m in members],
        li_variant=3, hllc_variant=2,  # 32 x 32 tiles, the fastest measured for requests of 256^2 and up
    )  # fmt: skip
    ens.set_targets([m.target for m in members])
    return ens


def _open_store(req: Request, st: State, out_dir: Path, morph) -> ZarrWriter:
    attrs = {"scheme": req.scheme, "dx": req.dx, "coarsen": 1,
             "units": {"depth": "m", "u": "m/s", "v": "m/s", "time": "s", "bed": "m"},
             "scenario": f"request {req.rid}", "request": {"rid": req.rid, "seed": req.seed, "side": req.side},
             "rain_type": "uniform", "rain_mm_hr": req.rain_mm_hr, "rain_duration_s": req.horizon,
             "end_time_s": req.horizon, "output_every_s": req.output_every, "solver": "rbsim serve (B200 CUDA)"}  # fmt: skip
    w = ZarrWriter(out_dir / f"req_{req.rid}.zarr", st.grid, 1 + len(output_times(req)), attrs,
                   bed_change=morph is not None)  # fmt: skip
    w.write_bed(st.z.cpu().numpy())
    return w


@dataclass
class Server:
    hbm_budget: float = 150e9
    graph_steps: int = 16
    device: str = "cuda"
    keep_depth: bool = False
    out_dir: str | None = None  # where requests with output_every > 0 get their result stores
    max_pending_frames: int = 8
    stats: dict = field(default_factory=dict)

    def run(self, requests: list[Request]) -> list[Result]:
        dev = torch.device(self.device)
        frames = FrameStream(dev, self.max_pending_frames) if self.out_dir is not None else None
        try:
            return self._serve(requests, dev, frames)
        finally:
            if frames is not None:
                frames.close()
                self.stats["frames"] = frames.frames

    def _serve(self, requests: list[Request], dev, frames: FrameStream | None) -> list[Result]:
        out_dir = Path(self.out_dir) if self.out_dir is not None else None
        if out_dir is not None:
            out_dir.mkdir(parents=True, exist_ok=True)
        queue = sorted(requests, key=lambda r: r.arrival)
        # the members of the current batch; a finished member stays in it (its clock has
        # stopped, its tiles return at once) until the batch is rebuilt, so a finish alone
        # costs no rebuild
        active: list[_Member] = []
        results: list[Result] = []
        used, replays, rebuilds = 0, 0, 0
        ens = None
        t0 = time.perf_counter()

        def drop_finished() -> None:
            nonlocal used, ens
            done = [m for m in active if m.done]
            if done:
                for m in done:
                    active.remove(m)
                    used -= m.nbytes
                ens = None

        while queue or any(not m.done for m in active):
            now = time.perf_counter() - t0
            if queue and queue[0].arrival <= now:
                drop_finished()  # the batch is rebuilt for the arrival anyway: free the finished first
            # admit, in arrival order, whatever has arrived and fits the budget
            while queue and queue[0].arrival <= now and used + request_bytes(queue[0]) <= self.hbm_budget:
                req = queue.pop(0)
                st, morph = build_state(req, dev)
                m = _Member(req, st, morph, admitted=time.perf_counter() - t0, nbytes=request_bytes(req),
                            next_act=req.morph_interval if morph is not None else math.inf)  # fmt: skip
                if frames is not None and req.output_every > 0.0:
                    m.writer = _open_store(req, st, out_dir, morph)
                    m.outputs = output_times(req)
                    frames.submit(m.writer, 0.0, m.frame_fields())
                active.append(m)
                used += m.nbytes
                ens = None
            live = [m for m in active if not m.done]
            if not live:
                drop_finished()
                if queue and queue[0].arrival <= now and request_bytes(queue[0]) > self.hbm_budget:
                    raise ValueError(f"request {queue[0].rid} needs {request_bytes(queue[0])} bytes, more than the "
                                     f"{self.hbm_budget:.0f}-byte budget")  # fmt: skip
                if queue:
                    time.sleep(max(0.0, min(queue[0].arrival - (time.perf_counter() - t0), 0.01)))
                continue
            if sum(m.req.side ** 2 for m in active if m.done) > sum(m.req.side ** 2 for m in live):
                drop_finished()  # finished members hold most of the batch's tiles: stop walking them
            if ens is None:
                ens = _build_ensemble(active, self.graph_steps)
                rebuilds += 1
            before = [m.steps for m in active]
            ens.replay()
            replays += 1
            clk = ens.read()
            if all(m.done or m.base_steps + c.steps == b for m, c, b in zip(active, clk, before, strict=True)):
                raise RuntimeError("the batch made no progress in a replay (every member's clock is inactive)")
            retarget = False
            for m, c in zip(active, clk, strict=True):
                if m.done:
                    continue
                m.t, m.steps = c.t, m.base_steps + c.steps
                if m.morph is not None and c.t >= m.next_act - EPS_T:
                    m.morph.advance(c.t, c.t - m.last_act)  # operator split, scheduler order
                    m.last_act = c.t
                    m.next_act += m.req.morph_interval
                    retarget = True
                if m.outputs and c.t >= m.outputs[0] - EPS_T:  # after the slow processes, as run.py
                    m.outputs.pop(0)
                    frames.submit(m.writer, c.t, m.frame_fields())
                    retarget = True
                if c.t >= m.req.horizon - EPS_T:
                    m.done = True
                    if m.writer is not None:
                        frames.finish(m.writer, {"steps": m.steps})
                    depth = m.st.h.cpu().numpy() if self.keep_depth else None
                    results.append(Result(m.req.rid, m.req.arrival, m.admitted, time.perf_counter() - t0, m.steps,
                                          m.t, depth))  # fmt: skip
            if retarget and ens is not None:
                ens.set_targets([m.target for m in active])
        wall = time.perf_counter() - t0
        lat = np.array([r.latency for r in results])
        self.stats = {
            "solves": len(results), "wall_s": wall, "solves_per_s": len(results) / wall if wall > 0 else 0.0,
            "p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
            "replays": replays, "ensemble_rebuilds": rebuilds,
        }  # fmt: skip
        return sorted(results, key=lambda r: r.rid)


def solve_alone(req: Request, device="cuda", graph_steps: int = 16, out_dir: str | None = None) -> Result:
    """One request on its own (the reference for "same alone and in the mix")."""
    srv = Server(graph_steps=graph_steps, device=device, keep_depth=True, out_dir=out_dir)
    r = Request(**{**req.__dict__, "arrival": 0.0})
    return srv.run([r])[0]


def serial_baseline(requests: list[Request], device="cuda", graph_steps: int = 16, out_dir: str | None = None) -> dict:
    """The plain loop: each request solved alone, in arrival order, one after another."""
    t0 = time.perf_counter()
    lat = []
    for req in sorted(requests, key=lambda r: r.arrival):
        now = time.perf_counter() - t0
        if req.arrival > now:
            time.sleep(req.arrival - now)
        solve_alone(req, device, graph_steps, out_dir)
        lat.append(time.perf_counter() - t0 - req.arrival)
    wall = time.perf_counter() - t0
    lat = np.array(lat)
    return {"solves": len(lat), "wall_s": wall, "solves_per_s": len(lat) / wall,
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99))}  # fmt: skip


def solve_per_step(req: Request, device="cuda", out_dir: str | None = None) -> int:
    """One request through the reference-shaped loop: the scheduler's ticks with a
    ``compute_dt`` (a device reduction read back every step) and a ``step`` launch per
    tick, slow processes and frames at their ticks (solver/run.py:369-398). Same state,
    forcing, sync times and step sequence as the server's device clock; returns the
    steps taken."""
    from .io.zarr_writer import AsyncFrameWriter
    from .scheduler import MultiRateScheduler
    from .schemes import get_scheme

    st, morph = build_state(req, torch.device(device))
    scheme = get_scheme(req.scheme)
    outs = output_times(req)
    frames = None
    if out_dir is not None and outs:
        Path(out_dir).mkdir(parents=True, exist_ok=True)
        writer = _open_store(req, st, Path(out_dir), morph)
        frames = AsyncFrameWriter(writer, st.device)
    member = _Member(req, st, morph, admitted=0.0, nbytes=0)

    def emit(t):
        f = member.frame_fields()
        frames.submit(t, f[0], f[1], f[2], f[3] if len(f) > 3 else None)

    if frames is not None:
        emit(0.0)
    sched = MultiRateScheduler(end_time=req.horizon, output_every=req.horizon, events=outs,
                               processes=[morph.as_slow_process()] if morph is not None else [])  # fmt: skip
    rain = req.rain_mm_hr / 3.6e6
    alpha = ALPHA[req.scheme]
    steps, pending = 0, list(outs)
    for tick in sched.ticks(lambda: scheme.compute_dt(st, alpha=alpha, dt_max=30.0)):
        scheme.step(st, dt=tick.dt, rain=rain if tick.t0 < req.horizon - EPS_T else 0.0, t=tick.t0)
        steps += 1
        for proc, elapsed in tick.due:
            proc.advance(tick.t1, elapsed)
        if pending and tick.t1 >= pending[0] - EPS_T:
            pending.pop(0)
            if frames is not None:
                emit(tick.t1)
    st.check_device_errors()
    if frames is not None:
        frames.close()
        frames.writer.finalize({"steps": steps})
    return steps


def serial_per_step_baseline(requests: list[Request], device="cuda", out_dir: str | None = None) -> dict:
    """The plain loop in the reference's shape: each request solved alone, in arrival
    order, one ``compute_dt`` + ``step`` per step (``solve_per_step``)."""
    t0 = time.perf_counter()
    lat = []
    for req in sorted(requests, key=lambda r: r.arrival):
        now = time.perf_counter() - t0
        if req.arrival > now:
            time.sleep(req.arrival - now)
        solve_per_step(req, device, out_dir)
        lat.append(time.perf_counter() - t0 - req.arrival)
    wall = time.perf_counter() - t0
    lat = np.array(lat)
    return {"solves": len(lat), "wall_s": wall, "solves_per_s": len(lat) / wall,
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99))}  # fmt: skip


def poisson_stream(rate: float, n: int, seed: int, side_lo: int = 256, side_hi: int = 4096,
                   horizon_lo: float = 600.0, horizon_hi: float = 7200.0) -> list[Request]:  # fmt: skip
    """Config-5 requests: Poisson arrivals, log-uniform sides, 70 % LI / 30 % HLLC, 10 % with Exner."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    for k in range(n):
        t += rng.exponential(1.0 / rate)
        side = int(round(math.exp(rng.uniform(math.log(side_lo), math.log(side_hi)))))
        scheme = "local_inertial" if rng.random() < 0.7 else "hllc_fv"
        exner = scheme == "local_inertial" and rng.random() < 0.1 / 0.7
        out.append(Request(rid=k, arrival=t, scheme=scheme, side=side,
                           horizon=float(rng.uniform(horizon_lo, horizon_hi)), seed=int(rng.integers(1 << 31)),
                           exner=exner, dx=10.0 if scheme == "local_inertial" else 2.0))  # fmt: skip
    return out
