"""Canonical Zarr v3 result store (the layout of solver/io/zarr_writer.py:1-154).

Layout (group ``results.zarr/``)::

    zarr.json       group metadata; attributes: scheme, dx, units, mass series, ...
    time            (T,)      float64  simulated seconds
    depth, u, v     (T, Y, X) float32  one chunk per frame
    bed             (Y, X)    float32  the initial bed
    bed_change      (T, Y, X) float32  cumulative bed change (morphology runs only)

Every array carries ``dimension_names`` so ``xarray.open_zarr`` opens it. The zarr
package is not a dependency: this module writes the Zarr v3 format directly
(``zarr.json`` metadata, the default ``c/i/j/k`` chunk keys, the little-endian
``bytes`` codec, no compression), which zarr-python 3 and xarray read.

``AsyncFrameWriter`` streams frames without stalling the solver: each frame's
fields are copied device-to-host on a side CUDA stream into pinned buffers and a
writer thread puts them on disk once the copy event completes.
"""

from __future__ import annotations

import json
import math
import os
import queue
import threading
from pathlib import Path

import numpy as np


def _json_safe(obj):
    if isinstance(obj, float) and not math.isfinite(obj):
        return "NaN" if math.isnan(obj) else ("Infinity" if obj > 0 else "-Infinity")
    if isinstance(obj, dict):
        return {str(k): _json_safe(v) for k, v in obj.items()}
    if isinstance(obj, (list, tuple)):
        return [_json_safe(v) for v in obj]
    if isinstance(obj, np.generic):
        return _json_safe(obj.item())
    return obj


def _atomic_write(path: Path, data: bytes) -> None:
    tmp = path.with_name(path.name + ".tmp")
    tmp.write_bytes(data)
    os.replace(tmp, path)


class _Array:
    def __init__(self, root: Path, name: str, shape, chunks, dtype: str, dims):
        self.path = root / name
        self.path.mkdir(parents=True, exist_ok=True)
        self.shape, self.chunks, self.dtype = tuple(shape), tuple(chunks), np.dtype(dtype).newbyteorder("<")
        meta = {
            "zarr_format": 3, "node_type": "array", "shape": list(self.shape),
            "data_type": {"f4": "float32", "f8": "float64"}[self.dtype.str[1:]],
            "chunk_grid": {"name": "regular", "configuration": {"chunk_shape": list(self.chunks)}},
            "chunk_key_encoding": {"name": "default", "configuration": {"separator": "/"}},
            "fill_value": 0.0, "codecs": [{"name": "bytes", "configuration": {"endian": "little"}}],
            "attributes": {}, "dimension_names": list(dims),
        }  # fmt: skip
        _atomic_write(self.path / "zarr.json", json.dumps(meta, indent=1).encode())

    def write_chunk(self, index: tuple, data: np.ndarray) -> None:
        arr = np.ascontiguousarray(data, dtype=self.dtype)
        if arr.shape != self.chunks:
            raise ValueError(f"{self.path.name}: chunk shape {arr.shape} != {self.chunks}")
        key = self.path.joinpath("c", *[str(i) for i in index])
        key.parent.mkdir(parents=True, exist_ok=True)
        _atomic_write(key, arr.tobytes())


class ZarrWriter:
    """Incremental writer preallocating ``n_frames`` along time (zarr_writer.py:33-154)."""

    def __init__(self, path, grid, n_frames: int, attrs: dict, *, bed_change: bool = False):
        self.path = Path(path)
        self.grid = grid
        self.n_frames = int(n_frames)
        self._i = 0
        self.path.mkdir(parents=True, exist_ok=True)
        ny, nx = grid.shape
        tyx = ("time", "y", "x")
        frame = (1, ny, nx)
        self._depth = _Array(self.path, "depth", (n_frames, ny, nx), frame, "f4", tyx)
        self._u = _Array(self.path, "u", (n_frames, ny, nx), frame, "f4", tyx)
        self._v = _Array(self.path, "v", (n_frames, ny, nx), frame, "f4", tyx)
        self._time = _Array(self.path, "time", (n_frames,), (n_frames,), "f8", ("time",))
        self._times = np.zeros(n_frames, np.float64)
        self._bed = _Array(self.path, "bed", (ny, nx), (ny, nx), "f4", ("y", "x"))
        self._bed_change = (_Array(self.path, "bed_change", (n_frames, ny, nx), frame, "f4", tyx)
                            if bed_change else None)  # fmt: skip
        self.attrs = dict(attrs)
        self._write_group()

    def _write_group(self) -> None:
        meta = {"zarr_format": 3, "node_type": "group", "attributes": _json_safe(self.attrs)}
        _atomic_write(self.path / "zarr.json", json.dumps(meta, indent=1).encode())

    def write_bed(self, bed: np.ndarray) -> None:
        self._bed.write_chunk((0, 0), bed)

    def write_static(self, name: str, field: np.ndarray) -> None:
        ny, nx = self.grid.shape
        _Array(self.path, name, (ny, nx), (ny, nx), "f4", ("y", "x")).write_chunk((0, 0), field)

    def append(self, time: float, depth, u, v, bed_change=None) -> None:
        """Write the next frame; ``bed_change`` exactly when the store carries it."""
        if self._i >= self.n_frames:
            raise IndexError(f"more frames than preallocated ({self.n_frames})")
        if (bed_change is None) != (self._bed_change is None):
            raise ValueError(
                "bed_change must be passed exactly when the store carries it; an omitted frame would "
                "store zeros, which reads as 'the bed did not move'"
            )
        i = self._i
        ny, nx = self.grid.shape
        self._depth.write_chunk((i, 0, 0), np.asarray(depth).reshape(1, ny, nx))
        self._u.write_chunk((i, 0, 0), np.asarray(u).reshape(1, ny, nx))
        self._v.write_chunk((i, 0, 0), np.asarray(v).reshape(1, ny, nx))
        if self._bed_change is not None:
            self._bed_change.write_chunk((i, 0, 0), np.asarray(bed_change, np.float32).reshape(1, ny, nx))
        self._times[i] = float(time)
        self._time.write_chunk((0,), self._times)
        self._i += 1

    @property
    def frames_written(self) -> int:
        return self._i

    def finalize(self, extra_attrs: dict | None = None) -> None:
        if extra_attrs:
            self.attrs.update(extra_attrs)
        self.attrs["n_frames"] = self._i
        if self._i < self.n_frames:
            self.attrs["n_frames_allocated"] = self.n_frames
        self._write_group()


def read_array(store, name: str) -> np.ndarray:
    """Read an array this writer produced (for tests and post-processing)."""
    root = Path(store) / name
    meta = json.loads((root / "zarr.json").read_text())
    dtype = np.dtype({"float32": "<f4", "float64": "<f8"}[meta["data_type"]])
    shape = tuple(meta["shape"])
    chunks = tuple(meta["chunk_grid"]["configuration"]["chunk_shape"])
    out = np.zeros(shape, dtype)
    grid = [range(-(-s // c)) for s, c in zip(shape, chunks, strict=True)]
    for idx in np.ndindex(*[len(g) for g in grid]):
        key = root.joinpath("c", *[str(i) for i in idx])
        if key.exists():
            block = np.frombuffer(key.read_bytes(), dtype).reshape(chunks)
            sl = tuple(slice(i * c, min((i + 1) * c, s)) for i, c, s in zip(idx, chunks, shape, strict=True))
            out[sl] = block[tuple(slice(0, s.stop - s.start) for s in sl)]
    return out


def _meta(store, name: str) -> dict:
    return json.loads((Path(store) / name / "zarr.json").read_text())


def has_array(store, name: str) -> bool:
    return (Path(store) / name / "zarr.json").is_file()


def array_shape(store, name: str) -> tuple:
    return tuple(_meta(store, name)["shape"])


def read_frame(store, name: str, index: int) -> np.ndarray:
    """Frame ``index`` of a (time, y, x) array written one frame per chunk; zeros
    (the fill value) where the frame was never written."""
    meta = _meta(store, name)
    _, ny, nx = meta["shape"]
    dtype = np.dtype({"float32": "<f4", "float64": "<f8"}[meta["data_type"]])
    key = Path(store) / name / "c" / str(int(index)) / "0" / "0"
    if not key.exists():
        return np.zeros((ny, nx), dtype)
    return np.frombuffer(key.read_bytes(), dtype).reshape(ny, nx)


def read_attrs(store) -> dict:
    return json.loads((Path(store) / "zarr.json").read_text())["attributes"]


class AsyncFrameWriter:
    """Frames copied D2H on a side stream into pinned buffers, written by a thread.

    ``submit`` records an event on the compute stream, makes the side stream wait
    for it, enqueues the copies there, and hands (event, buffers) to the writer
    thread, so the solver keeps stepping while the frame travels and hits disk.
    ``depth``/``u``/``v`` are device tensors (u and v already cell-centred).
    """

    def __init__(self, writer: ZarrWriter, device, slots: int = 3):
        import torch

        self.writer = writer
        self.device = device
        self._torch = torch
        self._side = torch.cuda.Stream(device)
        ny, nx = writer.grid.shape
        nfields = 4 if writer._bed_change is not None else 3
        self._free: queue.Queue = queue.Queue()
        for _ in range(slots):
            self._free.put([torch.empty((ny, nx), dtype=torch.float32, pin_memory=True) for _ in range(nfields)])
        self._jobs: queue.Queue = queue.Queue()
        self._error: BaseException | None = None
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._thread.start()

    def submit(self, time: float, depth, u, v, bed_change=None) -> None:
        if self._error is not None:
            raise self._error
        torch = self._torch
        bufs = self._free.get()
        # snapshot on the compute stream: the steps after this call write the state's
        # buffers again while the side stream may still be copying them
        srcs = [t.clone() for t in (depth, u, v)] + ([bed_change.float()] if bed_change is not None else [])
        ready = torch.cuda.Event()
        ready.record(torch.cuda.current_stream(self.device))
        self._side.wait_event(ready)
        with torch.cuda.stream(self._side):
            for b, s in zip(bufs, srcs, strict=True):
                b.copy_(s, non_blocking=True)
                s.record_stream(self._side)
            done = torch.cuda.Event()
            done.record(self._side)
        self._jobs.put((float(time), done, bufs, bed_change is not None))

    def _run(self) -> None:
        while True:
            job = self._jobs.get()
            if job is None:
                return
            time, done, bufs, has_bc = job
            try:
                done.synchronize()
                arrs = [b.numpy() for b in bufs]
                self.writer.append(time, arrs[0], arrs[1], arrs[2], arrs[3] if has_bc else None)
            except BaseException as e:  # surfaced on the next submit / close
                self._error = e
            finally:
                self._free.put(bufs)

    def close(self) -> None:
        self._jobs.put(None)
        self._thread.join()
        if self._error is not None:
            raise self._error
