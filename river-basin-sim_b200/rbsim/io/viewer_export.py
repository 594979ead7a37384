"""Viewer frame export: raw float32 tiles + ``manifest.json`` (the format of
solver/io/viewer_export.py:316-470).

A post-process over a finished result store (``rbsim.io.zarr_writer``): the
viewer cannot read Zarr, so each frame of one field is written as raw
little-endian float32, row-major with the store's orientation, and a manifest
tells the viewer where every byte went, what times the frames are at and which
colour range to use.

File format (kept byte- and key-compatible with the reference's reader):

* A frame that fits in one ``tile_size`` square is one file per frame,
  ``f0007_depth.raw``, listed under ``frames[i]["files"]``.
* A larger frame is cut into a row-major grid of tiles (edge tiles clipped),
  ``f0007_depth_r01_c02.raw``; the grid geometry is in ``manifest["tile_grid"]``
  once, and each frame lists its tile files in that order under
  ``frames[i]["tiles"]`` with an empty ``files``.
* ``manifest["static"]`` carries the bed the run stepped on (and the sub-grid
  channel width and depth when the store has them) through the same layout.
* ``manifest["global"][field]`` holds min / max / p50 / p99 over the wet cells of
  all frames (``max`` exact; the percentiles from a bounded, deterministic
  sample), each frame its own min / max.
* A morphology run declares that the exported terrain is its starting bed and by
  how much the run moved it; a channel run declares how far above the true water
  surface the viewer's drawn surface sits in-bank (``render_eta``).

Reads one frame at a time, so memory stays at a few frames whatever the run length.

    python -m rbsim.io.viewer_export results.zarr frames/ [--field depth] [--tile-size 512]
"""

from __future__ import annotations

import argparse
import json
import sys
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from ..channels import eta_from_h
from ..grid import H_DRY
from .zarr_writer import array_shape, has_array, read_array, read_attrs, read_frame

DEFAULT_TILE_SIZE = 512  # the store's chunk hint; a frame up to this size stays one file
PERCENTILE_SAMPLES = 4_000_000  # wet depths kept for the global percentiles, at most


def render_eta(h, z, w, d, dx: float) -> np.ndarray:
    """The water surface the viewer draws over a terrain without sub-grid trenches.

    Above bank full it is the storage curve itself, ``z + (h - h_bf)``; at or
    below bank full it is the bank, ``z`` (the true surface lies under the
    floodplain bed there, where the rendered terrain has nothing to show it in);
    a cell without a channel is ``z + h``. Continuous and monotone in ``h``.
    """
    h, z, w, d = (np.asarray(a, dtype=np.float64) for a in (h, z, w, d))
    channel = (w > 0.0) & (d > 0.0)
    bank_full = np.where(channel, w * d / dx, 0.0)
    return np.where(channel, z + np.maximum(h - bank_full, 0.0), z + h)


@dataclass(frozen=True)
class TileGrid:
    """Row-major tiles of ``size`` cells covering an ``(ny, nx)`` frame."""

    ny: int
    nx: int
    size: int

    @property
    def rows(self) -> int:
        return -(-self.ny // self.size)

    @property
    def cols(self) -> int:
        return -(-self.nx // self.size)

    @property
    def tiled(self) -> bool:
        return self.rows * self.cols > 1

    def tiles(self) -> list[dict]:
        s = self.size
        return [{"row": r, "col": c, "x": c * s, "y": r * s, "width": min(s, self.nx - c * s),
                 "height": min(s, self.ny - r * s)}
                for r in range(self.rows) for c in range(self.cols)]  # fmt: skip

    def describe(self) -> dict:
        return {"cols": self.cols, "rows": self.rows, "size": self.size, "tiles": self.tiles()}

    def write(self, arr: np.ndarray, out_dir: Path, *, key: str, stem: str) -> dict:
        """Write one field; return where it went (``files`` and, if tiled, ``tiles``)."""
        arr = np.ascontiguousarray(arr, dtype="<f4")
        if not self.tiled:
            name = f"{stem}.raw"
            (out_dir / name).write_bytes(arr.tobytes())
            return {"files": {key: name}}
        names = []
        for t in self.tiles():
            name = f"{stem}_r{t['row']:02d}_c{t['col']:02d}.raw"
            block = arr[t["y"]: t["y"] + t["height"], t["x"]: t["x"] + t["width"]]
            (out_dir / name).write_bytes(np.ascontiguousarray(block).tobytes())
            names.append(name)
        return {"files": {}, "tiles": {key: names}}


class _WetSample:
    """Wet values of every frame, thinned per frame to a bounded total."""

    def __init__(self, per_frame_cap: int):
        self.cap = max(int(per_frame_cap), 1)
        self.parts: list[np.ndarray] = []

    def add(self, wet: np.ndarray) -> None:
        step = -(-wet.size // self.cap) if wet.size > self.cap else 1
        self.parts.append(wet[::step].astype(np.float64, copy=False))

    def stats(self) -> dict:
        allw = np.concatenate(self.parts) if self.parts else np.empty(0)
        if allw.size == 0:
            return {"min": 0.0, "max": 0.0, "p50": 0.0, "p99": 0.0}
        p50, p99 = np.percentile(allw, [50.0, 99.0])
        return {"min": float(allw.min()), "max": float(allw.max()), "p50": float(p50), "p99": float(p99)}


class _InBankGap:
    """The largest height of the drawn surface above the true one over wet in-bank
    channel cells, with the frame where it occurred and that frame's in-bank count."""

    def __init__(self, bed: np.ndarray, w: np.ndarray, d: np.ndarray, dx: float, h_dry: float):
        self.bed, self.w, self.d, self.dx, self.h_dry = bed.astype(np.float64), w, d, dx, h_dry
        channel = (w > 0) & (d > 0)
        self.channel = channel
        self.bank_full = np.where(channel, w * d / dx, 0.0)
        self.worst = {"offset": 0.0, "cells": 0, "frame": -1}

    def add(self, i: int, h: np.ndarray) -> None:
        in_bank = self.channel & (h >= self.h_dry) & (h <= self.bank_full)
        if not in_bank.any():
            return
        gap = (render_eta(h, self.bed, self.w, self.d, self.dx)
               - eta_from_h(h, self.bed, self.w, self.d, self.dx))[in_bank]  # fmt: skip
        top = float(gap.max())
        if top > self.worst["offset"]:
            self.worst = {"offset": top, "cells": int(in_bank.sum()), "frame": i}

    def note(self) -> dict:
        return {"cells": int(self.channel.sum()), "width_max_m": float(self.w.max()),
                "depth_max_m": float(self.d.max()), "dx_m": float(self.dx),
                "in_bank_offset_m": self.worst["offset"], "in_bank_cells": self.worst["cells"],
                "frame": self.worst["frame"],
                "note": "water below bank full is drawn at the bank: its true surface is under the floodplain bed "
                        "and the rendered terrain carries no sub-grid trench"}  # fmt: skip


def export_frames(store, out_dir, *, field: str = "depth", h_dry: float = H_DRY,
                  tile_size: int = DEFAULT_TILE_SIZE) -> Path:  # fmt: skip
    """Export ``field`` of a result store as per-frame raw tiles; returns the manifest path."""
    store, out_dir = Path(store), Path(out_dir)
    out_dir.mkdir(parents=True, exist_ok=True)
    attrs = read_attrs(store)
    n_alloc, ny, nx = array_shape(store, field)
    n_frames = min(int(attrs.get("n_frames", n_alloc)), n_alloc)  # frames actually written
    times = read_array(store, "time")
    dx = float(attrs.get("dx", 1.0))
    grid = TileGrid(ny, nx, max(int(tile_size), 1))

    channels = None
    if has_array(store, "channel_width") and has_array(store, "channel_depth"):
        channels = (read_array(store, "channel_width").astype("<f4"), read_array(store, "channel_depth").astype("<f4"))
    bed = read_array(store, "bed") if has_array(store, "bed") else None
    gap = _InBankGap(bed, *channels, dx, h_dry) if channels is not None and field == "depth" and bed is not None \
        else None  # fmt: skip

    sample = _WetSample(PERCENTILE_SAMPLES)
    frames, top = [], 0.0
    for i in range(n_frames):
        arr = read_frame(store, field, i).astype("<f4", copy=False)
        entry = {"index": i, "time": float(times[i])}
        entry.update(grid.write(arr, out_dir, key=field, stem=f"f{i:04d}_{field}"))
        lo, hi = float(arr.min()), float(arr.max())
        entry[field] = {"min": lo, "max": hi}
        frames.append(entry)
        top = max(top, hi)
        sample.add(arr[arr >= h_dry])
        if gap is not None:
            gap.add(i, arr)
    glob = sample.stats()
    glob["max"] = top  # exact, whatever the percentile sample kept

    manifest = {
        "dx": dx, "crs": str(attrs.get("crs", "")), "scheme": str(attrs.get("scheme", "")),
        "coarsen": int(attrs.get("coarsen", 1)), "grid": {"width": nx, "height": ny},
        "tile_grid": grid.describe(), "fields": [field], "h_dry": float(h_dry), "n_frames": n_frames,
        "global": {field: glob}, "frames": frames,
    }  # fmt: skip
    if bed is not None:
        static = grid.write(bed, out_dir, key="bed", stem="bed")
        names = ["bed"]
        for name, arr in zip(("channel_width", "channel_depth"), channels or (), strict=False):
            part = grid.write(arr, out_dir, key=name, stem=name)
            static["files"].update(part["files"])
            if "tiles" in part:
                static.setdefault("tiles", {}).update(part["tiles"])
            names.append(name)
        static["fields"] = names
        static["bed"] = {"min": float(bed.min()), "max": float(bed.max())}
        if gap is not None:
            static["channel"] = gap.note()
        manifest["static"] = static
    if has_array(store, "bed_change") and n_frames > 0:
        last = n_frames - 1
        dz = read_frame(store, "bed_change", last).astype(np.float64)
        manifest["morphology"] = {
            "bed_change": {"min": float(dz.min()), "max": float(dz.max()), "frame": last, "time": float(times[last])},
            "static_bed": "initial",
            "note": "terrain is the bed at t=0; this run moved it (see bed_change in the result store); the viewer "
                    "does not animate terrain",
        }  # fmt: skip
    if isinstance(attrs.get("domain"), dict):
        manifest["domain"] = dict(attrs["domain"])
    path = out_dir / "manifest.json"
    path.write_text(json.dumps(manifest, indent=2), encoding="utf-8")
    return path


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m rbsim.io.viewer_export",
                                 description="Export per-frame viewer tiles from a result store.")  # fmt: skip
    ap.add_argument("store")
    ap.add_argument("out_dir")
    ap.add_argument("--field", default="depth")
    ap.add_argument("--tile-size", type=int, default=DEFAULT_TILE_SIZE)
    args = ap.parse_args(argv)
    print(f"viewer export: {export_frames(args.store, args.out_dir, field=args.field, tile_size=args.tile_size)}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
