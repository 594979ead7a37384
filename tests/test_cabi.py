"""The C ABI library loads without a GPU and exports every entry point of include/rbsim.h."""

from __future__ import annotations

import ctypes
import os
import re

import pytest
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# The refusal tests below hand the library made-up device addresses and rely on its
# argument checks refusing before any launch. They run only where no CUDA device is
# visible, so that a check that ever stopped refusing could not launch a kernel on them.
no_device = pytest.mark.skipif(torch.cuda.is_available(), reason="made-up device addresses: host-only machines")
HEADERS = [os.path.join(ROOT, "include", "rbsim.h")]


def declared_functions(path):
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(rb_[a-z0-9_]+)\s*\(", text, flags=re.M)))


def _lib():
    import build  # river-basin-sim_b200/build.py

    build.build()
    from rbsim import _lib

    return _lib.lib()


def test_every_declared_entry_point_is_exported():
    L = _lib()
    names = [n for h in HEADERS for n in declared_functions(h)]
    assert len(names) >= 15, names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, f"declared in include/ but not exported: {missing}"


def test_binding_table_covers_the_header():
    from rbsim import _lib

    names = [n for h in HEADERS for n in declared_functions(h)]
    assert sorted(_lib.SIGNATURES) == sorted(names)


def test_struct_layouts_match_the_c_compiler(tmp_path):
    """The ctypes mirrors have exactly the layout gcc gives the header's structs."""
    import subprocess

    from rbsim import _lib

    structs = {"rb_li_fields": _lib.LiFields, "rb_hllc_fields": _lib.HllcFields, "rb_step_args": _lib.StepArgs,
               "rb_clock_config": _lib.ClockConfig, "rb_clock_state": _lib.ClockState,
               "rb_ensemble_layout": _lib.EnsembleLayout}  # fmt: skip
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "rbsim.h"', "int main(void) {"]
    for cname, cls in structs.items():
        lines.append(f'  printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'  printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("  return 0;\n}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                       check=True).stdout.splitlines())
    for cname, cls in structs.items():
        assert int(got[cname]) == ctypes.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(cls, fname).offset, f"{cname}.{fname}"


def test_host_only_calls_work_without_a_device():
    L = _lib()
    assert L.rb_li_workspace_bytes(2048, 2048) > 0
    assert L.rb_hllc_workspace_bytes(2048, 2048) > 3 * 2048 * 2048 * 4
    assert L.rb_li_workspace_bytes(0, 5) == 0
    major, minor, arch = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
    assert L.rb_version(ctypes.byref(major), ctypes.byref(minor), ctypes.byref(arch)) == 0
    assert arch.value == 100


@no_device
def test_argument_errors_are_reported_without_touching_the_device():
    from rbsim import _lib

    L = _lib.lib()
    f = _lib.LiFields()
    f.ny, f.nx, f.dx = 0, 4, 1.0
    a = _lib.StepArgs(1.0, 0.0, 1.0, 1, 0)
    rc = L.rb_li_step(ctypes.byref(f), 0, ctypes.byref(a), ctypes.c_void_p(1), None)
    assert rc == _lib.RB_ERR_ARG
    assert "grid 0 x 4" in _lib.last_error()
    f.ny = 4
    a.dt = -1.0
    f.bc[:] = [0, 0, 0, 0]
    rc = L.rb_li_step(ctypes.byref(f), 0, ctypes.byref(a), ctypes.c_void_p(1), None)
    assert rc == _lib.RB_ERR_STEP
    try:
        _lib.check(rc)
    except RuntimeError as e:
        assert "non-positive timestep" in str(e)
    f.bc[:] = [2, 0, 0, 0]
    a.dt = 1.0
    assert L.rb_li_step(ctypes.byref(f), 0, ctypes.byref(a), ctypes.c_void_p(1), None) == _lib.RB_ERR_ARG


def test_ensemble_layout_counts_each_variants_tiles():
    """Host only: the ensemble layout sizes its work lists from the chosen tile shapes
    (LI 32x16 / 32x8 / 64x8 / 32x32, HLLC 32x16 / 32x8 / 32x32) and refuses others."""
    from rbsim import _lib

    L = _lib.lib()
    scheme = (ctypes.c_int32 * 3)(0, 1, 1)
    ny = (ctypes.c_int32 * 3)(100, 70, 33)
    nx = (ctypes.c_int32 * 3)(64, 65, 1)

    def tiles(n_y, n_x, tx, ty):
        return -(-n_x // tx) * -(-n_y // ty)

    li_shapes = {0: (32, 16), 1: (32, 8), 2: (64, 8), 3: (32, 32)}
    hllc_shapes = {0: (32, 16), 1: (32, 8), 2: (32, 32)}
    for lv, (ltx, lty) in li_shapes.items():
        for hv, (htx, hty) in hllc_shapes.items():
            out = _lib.EnsembleLayout()
            assert L.rb_ensemble_layout_make(3, scheme, ny, nx, lv, hv, ctypes.byref(out)) == 0
            assert (out.n_li, out.n_hllc) == (1, 2)
            assert out.li_tiles == tiles(100, 64, ltx, lty)
            assert out.hllc_tiles == tiles(70, 65, htx, hty) + tiles(33, 1, htx, hty)
            assert out.bytes > 0
    out = _lib.EnsembleLayout()
    assert L.rb_ensemble_layout_make(3, scheme, ny, nx, 0, 3, ctypes.byref(out)) == _lib.RB_ERR_ARG
    assert "unknown tile variant" in _lib.last_error()
    assert L.rb_ensemble_layout_make(3, scheme, ny, nx, 4, 0, ctypes.byref(out)) == _lib.RB_ERR_ARG


@no_device
def test_both_hllc_step_entry_points_refuse_the_same_inputs_without_a_device():
    """rb_hllc_step and rb_hllc_step_noalloc apply the same argument checks, all before
    any device call: each case below carries exactly one defect on otherwise valid
    arguments (the buffer addresses are never dereferenced on the host)."""
    from rbsim import _lib

    L = _lib.lib()

    def fields(ny=64, nx=48):
        f = _lib.HllcFields()
        f.ny, f.nx, f.dx = ny, nx, 2.0
        for k, name in enumerate(("h", "hu", "hv")):
            getattr(f, name)[0], getattr(f, name)[1] = 4096 * (2 * k + 1), 4096 * (2 * k + 2)
        f.z, f.n = 4096 * 7, 4096 * 8
        f.bc[:] = [0, 1, 2, 0]
        return f

    def args(dt=0.5):
        return _lib.StepArgs(dt, 0.0, 1.0, 1, 0)

    def both(f, a, cur=0):
        ws = ctypes.c_void_p(4096 * 16)
        return (L.rb_hllc_step(f if f is None else ctypes.byref(f), cur, ctypes.byref(a), ws, None),
                L.rb_hllc_step_noalloc(f if f is None else ctypes.byref(f), cur, ctypes.byref(a), None, None))

    cases = []
    cases.append(("null fields", both(None, args()), _lib.RB_ERR_ARG))
    f = fields(0, 48)
    cases.append(("empty grid", both(f, args()), _lib.RB_ERR_ARG))
    f = fields()
    f.dx = float("inf")
    cases.append(("infinite dx", both(f, args()), _lib.RB_ERR_ARG))
    cases.append(("infinite dt", both(fields(), args(float("inf"))), _lib.RB_ERR_STEP))
    cases.append(("nan dt", both(fields(), args(float("nan"))), _lib.RB_ERR_STEP))
    cases.append(("zero dt", both(fields(), args(0.0)), _lib.RB_ERR_STEP))
    f = fields()
    f.bc[2] = 7
    cases.append(("unknown edge kind", both(f, args()), _lib.RB_ERR_ARG))
    cases.append(("cur 2", both(fields(), args(), cur=2), _lib.RB_ERR_ARG))
    f = fields()
    f.hv[1] = None
    cases.append(("missing buffer", both(f, args()), _lib.RB_ERR_ARG))
    for what, got, want in cases:
        assert got == (want, want), what
    f = fields(1025, 1024)
    assert L.rb_hllc_step_noalloc(ctypes.byref(f), 0, ctypes.byref(args()), None, None) == _lib.RB_ERR_ARG
    assert "1048576-cell" in _lib.last_error()


@no_device
def test_clock_start_refuses_bad_configs_without_a_device():
    """The device clock's start checks its configuration before reading it: a null
    config (with a fixed_stage edge, whose stage curve the HLLC start looks up), a bad
    buffer index, a missing sync array, non-positive alpha or dt_max, point sources
    without their tables, and a fixed_stage edge without a stage curve."""
    from rbsim import _lib

    L = _lib.lib()
    ws = ctypes.c_void_p(4096 * 16)
    f = _lib.HllcFields()
    f.ny, f.nx, f.dx = 32, 32, 1.0
    for k, name in enumerate(("h", "hu", "hv")):
        getattr(f, name)[0], getattr(f, name)[1] = 4096 * (2 * k + 1), 4096 * (2 * k + 2)
    f.z, f.n = 4096 * 7, 4096 * 8
    f.bc[:] = [0, 0, 2, 0]  # east fixed_stage
    assert L.rb_hllc_clock_start(ctypes.byref(f), 0, None, ws, None) == _lib.RB_ERR_ARG
    assert "null config" in _lib.last_error()

    def cfg(**kw):
        c = _lib.ClockConfig()
        c.alpha, c.dt_max, c.nsync = 0.45, 5.0, 0
        c.stage_off[:] = [0, 0, 0, 2, 2]  # two knots for edge 2 (east)
        for k, v in kw.items():
            setattr(c, k, v)
        return c

    for bad in (dict(nsync=3), dict(alpha=0.0), dict(dt_max=-1.0), dict(nsrc=2)):
        assert L.rb_hllc_clock_start(ctypes.byref(f), 0, ctypes.byref(cfg(**bad)), ws, None) == _lib.RB_ERR_ARG, bad
    assert L.rb_hllc_clock_start(ctypes.byref(f), 2, ctypes.byref(cfg()), ws, None) == _lib.RB_ERR_ARG
    no_curve = cfg()
    no_curve.stage_off[:] = [0, 0, 0, 0, 0]
    assert L.rb_hllc_clock_start(ctypes.byref(f), 0, ctypes.byref(no_curve), ws, None) == _lib.RB_ERR_ARG
    assert "no stage curve" in _lib.last_error()
    li = _lib.LiFields()
    li.ny, li.nx, li.dx = 32, 32, 1.0
    for k, name in enumerate(("h", "qx", "qy")):
        getattr(li, name)[0], getattr(li, name)[1] = 4096 * (2 * k + 1), 4096 * (2 * k + 2)
    li.z, li.n = 4096 * 7, 4096 * 8
    assert L.rb_li_clock_start(ctypes.byref(li), 0, None, ws, None) == _lib.RB_ERR_ARG


def _fake_li(ny, nx):
    from rbsim import _lib

    f = _lib.LiFields()
    f.ny, f.nx, f.dx = ny, nx, 10.0
    for k, name in enumerate(("h", "qx", "qy")):
        getattr(f, name)[0], getattr(f, name)[1] = 4096 * (2 * k + 1), 4096 * (2 * k + 2)
    f.z, f.n = 4096 * 7, 4096 * 8
    return f


def _fake_hllc(ny, nx):
    from rbsim import _lib

    f = _lib.HllcFields()
    f.ny, f.nx, f.dx = ny, nx, 10.0
    for k, name in enumerate(("h", "hu", "hv")):
        getattr(f, name)[0], getattr(f, name)[1] = 4096 * (2 * k + 1), 4096 * (2 * k + 2)
    f.z, f.n = 4096 * 7, 4096 * 8
    return f


@no_device
def test_compute_dt_refuses_a_missing_current_buffer():
    """A null current depth (or momentum) buffer is an argument error, not a kernel launch on NULL."""
    from rbsim import _lib

    L = _lib.lib()
    ws, dt = ctypes.c_void_p(4096 * 16), ctypes.c_double()
    li = _fake_li(8, 8)
    li.h[1] = None
    assert L.rb_li_compute_dt(ctypes.byref(li), 1, 0.7, 5.0, ws, None, ctypes.byref(dt)) == _lib.RB_ERR_ARG
    assert "missing depth buffer" in _lib.last_error()
    hl = _fake_hllc(8, 8)
    hl.hu[0] = None
    assert L.rb_hllc_compute_dt(ctypes.byref(hl), 0, 0.45, 5.0, ws, None, ctypes.byref(dt)) == _lib.RB_ERR_ARG
    assert "missing state buffer" in _lib.last_error()


@no_device
def test_ensemble_init_refuses_a_layout_that_does_not_fit_its_domains():
    """rb_ensemble_init sizes host vectors and device areas from the layout, so it checks
    the layout against the scheme array, the buffer indices and the domains' tiles first."""
    from rbsim import _lib

    L = _lib.lib()
    n = 3
    scheme = (ctypes.c_int32 * n)(0, 1, 1)
    ny = (ctypes.c_int32 * n)(40, 30, 20)
    nx = (ctypes.c_int32 * n)(40, 30, 20)
    lay = _lib.EnsembleLayout()
    assert L.rb_ensemble_layout_make(n, scheme, ny, nx, 0, 0, ctypes.byref(lay)) == 0
    li = (_lib.LiFields * 1)(_fake_li(40, 40))
    hl = (_lib.HllcFields * 2)(_fake_hllc(30, 30), _fake_hllc(20, 20))
    wss = (ctypes.c_void_p * n)(4096 * 32, 4096 * 48, 4096 * 64)
    cfgs = (_lib.ClockConfig * n)()
    for c in cfgs:
        c.alpha, c.dt_max = 0.5, 5.0
    cur = (ctypes.c_int32 * n)(0, 1, 0)
    ens = ctypes.c_void_p(4096 * 128)

    def init(layout, sch=scheme, cr=cur, hls=hl):
        return L.rb_ensemble_init(ctypes.byref(layout), ens, sch, li, hls, wss, cfgs, cr, None)

    assert init(lay, sch=(ctypes.c_int32 * n)(0, 0, 1)) == _lib.RB_ERR_ARG
    assert "does not match the layout" in _lib.last_error()
    assert init(lay, cr=(ctypes.c_int32 * n)(0, 2, 0)) == _lib.RB_ERR_ARG
    assert "cur must be 0 or 1" in _lib.last_error()
    forged = _lib.EnsembleLayout.from_buffer_copy(lay)
    forged.n_li = 5
    assert init(forged) == _lib.RB_ERR_ARG
    assert "not one rb_ensemble_layout_make made" in _lib.last_error()
    bigger = (_lib.HllcFields * 2)(_fake_hllc(300, 300), _fake_hllc(20, 20))
    assert init(_lib.EnsembleLayout.from_buffer_copy(lay), hls=bigger) == _lib.RB_ERR_ARG
    assert "more tiles than the layout" in _lib.last_error()
