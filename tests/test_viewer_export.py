"""Viewer frame export (solver/io/test_viewer_export.py): raw tiles reload to the store's
frames byte for byte, the manifest's ranges and geometry are right, and the static bed,
channel geometry and morphology notes ride along. CPU only: the stores are written with
the package's own Zarr writer from synthetic frames."""

from __future__ import annotations

import json

import numpy as np
import pytest

from rbsim.channels import eta_from_h
from rbsim.grid import Grid
from rbsim.io.viewer_export import export_frames, main, render_eta
from rbsim.io.zarr_writer import ZarrWriter, read_array


def _store(tmp_path, *, ny=16, nx=20, frames=4, written=None, channels=None, morphology=False, attrs=None,
           name="r.zarr"):  # fmt: skip
    """A result store of ``frames`` frames of a filling basin (non-square: catches a transpose)."""
    rng = np.random.default_rng(3)
    yy, xx = np.mgrid[0:ny, 0:nx]
    bed = (((yy - ny / 2) ** 2 + (xx - nx / 2) ** 2) * 0.02).astype(np.float32)
    grid = Grid(ny=ny, nx=nx, dx=20.0)
    base = {"scheme": "local_inertial", "dx": 20.0, "coarsen": 1, **(attrs or {})}
    w = ZarrWriter(tmp_path / name, grid, frames, base, bed_change=morphology)
    w.write_bed(bed)
    if channels is not None:
        w.write_static("channel_width", channels[0])
        w.write_static("channel_depth", channels[1])
    for i in range(frames if written is None else written):
        depth = np.maximum(0.3 * i - 0.05 * bed + 0.01 * rng.random((ny, nx)), 0.0).astype(np.float32)
        dz = (-0.01 * i * rng.random((ny, nx))).astype(np.float32) if morphology else None
        w.append(200.0 * i, depth, depth * 0.1, depth * 0.2, dz)
    w.finalize({})
    return tmp_path / name, bed


def test_frames_roundtrip_store_bytes(tmp_path):
    store, _ = _store(tmp_path)
    out = tmp_path / "frames"
    export_frames(store, out)
    depth = read_array(store, "depth")
    m = json.loads((out / "manifest.json").read_text())
    assert m["n_frames"] == 4 and m["fields"] == ["depth"] and m["grid"] == {"width": 20, "height": 16}
    assert (m["tile_grid"]["cols"], m["tile_grid"]["rows"]) == (1, 1)
    assert "tiles" not in m["frames"][0]
    for fr in m["frames"]:
        raw = np.fromfile(out / fr["files"]["depth"], dtype="<f4").reshape(16, 20)
        assert np.array_equal(raw, depth[fr["index"]])
        assert fr["depth"] == {"min": float(depth[fr["index"]].min()), "max": float(depth[fr["index"]].max())}
        assert fr["time"] == 200.0 * fr["index"]


def test_global_stats_are_robust_and_exact_at_the_top(tmp_path):
    store, _ = _store(tmp_path)
    out = tmp_path / "frames"
    export_frames(store, out)
    g = json.loads((out / "manifest.json").read_text())["global"]["depth"]
    depth = read_array(store, "depth")
    wet = depth[depth >= 1e-3].astype(np.float64)
    assert g["max"] == float(depth.max())
    assert g["p50"] == pytest.approx(float(np.percentile(wet, 50.0)))
    assert g["p99"] == pytest.approx(float(np.percentile(wet, 99.0)))
    assert 0.0 <= g["min"] <= g["p50"] <= g["p99"] <= g["max"]


def test_only_written_frames_are_exported(tmp_path):
    store, _ = _store(tmp_path, frames=5, written=3)
    out = tmp_path / "frames"
    m = json.loads(export_frames(store, out).read_text())
    assert m["n_frames"] == 3 and len(m["frames"]) == 3
    assert not (out / "f0003_depth.raw").exists()


def test_large_frames_split_into_a_tile_grid_that_reassembles(tmp_path):
    store, bed = _store(tmp_path, ny=12, nx=20)
    out = tmp_path / "frames"
    m = json.loads(export_frames(store, out, tile_size=8).read_text())
    grid = m["tile_grid"]
    assert (grid["rows"], grid["cols"], grid["size"]) == (2, 3, 8)
    assert [t["width"] for t in grid["tiles"][:3]] == [8, 8, 4]
    assert [t["height"] for t in grid["tiles"][::3]] == [8, 4]
    assert sum(t["width"] * t["height"] for t in grid["tiles"]) == 12 * 20
    depth = read_array(store, "depth")
    for fr in m["frames"]:
        assert fr["files"] == {}
        names = fr["tiles"]["depth"]
        assert len(names) == len(grid["tiles"])
        rebuilt = np.zeros((12, 20), np.float32)
        for t, name in zip(grid["tiles"], names, strict=True):
            block = np.fromfile(out / name, dtype="<f4").reshape(t["height"], t["width"])
            rebuilt[t["y"]: t["y"] + t["height"], t["x"]: t["x"] + t["width"]] = block
        assert np.array_equal(rebuilt, depth[fr["index"]])
    static = m["static"]
    assert static["files"] == {} and len(static["tiles"]["bed"]) == 6
    rebuilt = np.zeros_like(bed)
    for t, name in zip(grid["tiles"], static["tiles"]["bed"], strict=True):
        rebuilt[t["y"]: t["y"] + t["height"], t["x"]: t["x"] + t["width"]] = np.fromfile(
            out / name, dtype="<f4").reshape(t["height"], t["width"])  # fmt: skip
    assert np.array_equal(rebuilt, bed)


def test_static_bed_ships_with_the_frames(tmp_path):
    store, bed = _store(tmp_path)
    out = tmp_path / "frames"
    m = json.loads(export_frames(store, out).read_text())
    static = m["static"]
    assert static["fields"] == ["bed"] and list(static["files"]) == ["bed"]
    got = np.fromfile(out / static["files"]["bed"], dtype="<f4").reshape(bed.shape)
    assert np.array_equal(got, bed)
    assert static["bed"] == {"min": float(bed.min()), "max": float(bed.max())}
    assert "channel" not in static and "morphology" not in m
    assert not any("channel" in p.name or "bed_change" in p.name for p in out.iterdir())


def test_manifest_carries_the_domain_record(tmp_path):
    store, _ = _store(tmp_path, attrs={"coarsen": 2, "domain": {"gap_cells": 7, "fill_value": 12.5}})
    m = json.loads(export_frames(store, tmp_path / "frames").read_text())
    assert m["coarsen"] == 2 and m["domain"] == {"gap_cells": 7, "fill_value": 12.5}


def test_a_morphology_run_declares_its_terrain_is_the_starting_bed(tmp_path):
    store, bed = _store(tmp_path, morphology=True)
    out = tmp_path / "frames"
    m = json.loads(export_frames(store, out).read_text())
    final = read_array(store, "bed_change")[-1]
    morph = m["morphology"]
    assert morph["static_bed"] == "initial"
    assert morph["bed_change"]["min"] == float(final.min()) < 0.0
    assert morph["bed_change"]["max"] == float(final.max())
    assert morph["bed_change"]["frame"] == 3 and morph["bed_change"]["time"] == 600.0
    assert np.array_equal(np.fromfile(out / "bed.raw", dtype="<f4").reshape(bed.shape), bed)
    assert not any("bed_change" in p.name for p in out.iterdir())


def test_drawn_surface_is_the_storage_curve_overbank_and_the_bank_below():
    dx = 20.0
    z = np.full(6, 10.0)
    w = np.full(6, 8.0)
    d = np.full(6, 1.0)
    h_bf = 8.0 * 1.0 / dx
    h = np.array([0.0, 0.1, 0.3, h_bf, h_bf + 1e-3, 1.0])
    drawn = render_eta(h, z, w, d, dx)
    true = eta_from_h(h, z, w, d, dx)
    over = h > h_bf
    assert np.array_equal(drawn[over], true[over])
    assert np.all(drawn[~over] == z[~over])
    assert np.all(drawn >= true - 1e-12)
    assert drawn[1] - true[1] == pytest.approx(d[1] - h[1] * dx / w[1], rel=1e-12)
    zeros = np.zeros(3)
    hh, zz = np.array([0.0, 0.5, 2.0]), np.array([1.0, 2.0, 3.0])
    assert np.array_equal(render_eta(hh, zz, zeros, zeros, dx), zz + hh)
    assert np.array_equal(render_eta(hh, zz, np.full(3, 8.0), zeros, dx), zz + hh)


def test_channel_geometry_ships_and_the_in_bank_offset_is_measured(tmp_path):
    ny, nx, dx = 16, 20, 20.0
    w = np.zeros((ny, nx), np.float32)
    d = np.zeros((ny, nx), np.float32)
    w[:, 7] = 8.0
    d[:, 7] = 1.0
    store, bed = _store(tmp_path, channels=(w, d))
    out = tmp_path / "frames"
    m = json.loads(export_frames(store, out, tile_size=8).read_text())
    static = m["static"]
    assert static["fields"] == ["bed", "channel_width", "channel_depth"]
    assert len(static["tiles"]["channel_width"]) == len(m["tile_grid"]["tiles"])
    chan = static["channel"]
    assert chan["cells"] == 16 and chan["width_max_m"] == 8.0 and chan["depth_max_m"] == 1.0 and chan["dx_m"] == dx
    depth = read_array(store, "depth")
    has = (w > 0) & (d > 0)
    h_bf = np.where(has, w * d / dx, 0.0)
    best = (0.0, 0, -1)
    for i, h in enumerate(depth):
        in_bank = has & (h >= 1e-3) & (h <= h_bf)
        if in_bank.any():
            gap = (render_eta(h, bed, w, d, dx) - eta_from_h(h, bed, w, d, dx))[in_bank].max()
            if gap > best[0]:
                best = (float(gap), int(in_bank.sum()), i)
    assert best[1] > 0, "the fixture must wet the channel below bank full somewhere"
    assert (chan["in_bank_offset_m"], chan["in_bank_cells"], chan["frame"]) == (pytest.approx(best[0]), best[1],
                                                                                best[2])  # fmt: skip
    assert 0.0 < chan["in_bank_offset_m"] <= chan["depth_max_m"]


def test_cli_entry_point(tmp_path):
    store, _ = _store(tmp_path)
    assert main([str(store), str(tmp_path / "cli")]) == 0
    assert (tmp_path / "cli" / "manifest.json").exists()


def _reassemble(out, tiles, names, shape):
    full = np.zeros(shape, np.float32)
    for t, name in zip(tiles, names, strict=True):
        block = np.fromfile(out / name, dtype="<f4").reshape(t["height"], t["width"])
        full[t["y"] : t["y"] + t["height"], t["x"] : t["x"] + t["width"]] = block
    return full


def test_static_fields_are_tiled_with_the_frame_layout(tmp_path):
    """solver/io/test_viewer_export.py:149, :371: in a tiled export the bed and the channel
    geometry ride the frames' tile grid, so one reader decodes all of them."""
    ny, nx = 16, 20
    w = np.zeros((ny, nx), np.float32)
    d = np.zeros((ny, nx), np.float32)
    w[:, nx // 2], d[:, nx // 2] = 8.0, 1.0
    store, bed = _store(tmp_path, ny=ny, nx=nx, channels=(w, d))
    out = tmp_path / "tiled"
    manifest = json.loads(export_frames(store, out, tile_size=8).read_text())
    tiles = manifest["tile_grid"]["tiles"]
    static = manifest["static"]
    assert static["files"] == {} and len(tiles) > 1
    for name, want in (("bed", bed), ("channel_width", w), ("channel_depth", d)):
        assert np.array_equal(_reassemble(out, tiles, static["tiles"][name], (ny, nx)), want), name


def test_a_still_bed_and_a_channel_free_run_add_nothing_to_the_manifest(tmp_path):
    """solver/io/test_viewer_export.py:258, :435: no morphology note, no channel keys or files."""
    store, _ = _store(tmp_path)
    out = tmp_path / "f"
    manifest = json.loads(export_frames(store, out).read_text())
    assert "morphology" not in manifest
    static = manifest["static"]
    assert static["fields"] == ["bed"] and "channel" not in static and list(static["files"]) == ["bed"]
    assert not any("channel" in p.name for p in out.iterdir())


def test_a_cell_without_a_channel_is_drawn_exactly_as_before():
    """solver/io/test_viewer_export.py:327: z + h bit for bit, also for half a channel."""
    z = np.array([1.0, 250.0, -3.5])
    h = np.array([0.0, 0.001, 2.25])
    zeros = np.zeros(3)
    assert np.array_equal(render_eta(h, z, zeros, zeros, 20.0), z + h)
    assert np.array_equal(render_eta(h, z, np.full(3, 8.0), zeros, 20.0), z + h)
    assert np.array_equal(render_eta(h, z, zeros, np.full(3, 1.0), 20.0), z + h)


def test_one_tile_exports_the_same_bytes_whatever_the_tile_size(tmp_path):
    """solver/io/test_viewer_export.py:449: a frame that fits one tile is written identically."""
    store, _ = _store(tmp_path)
    a, b = tmp_path / "a", tmp_path / "b"
    export_frames(store, a)
    export_frames(store, b, tile_size=4096)
    for fr in json.loads((a / "manifest.json").read_text())["frames"]:
        name = fr["files"]["depth"]
        assert (a / name).read_bytes() == (b / name).read_bytes()
