"""rb_hllc_step_noalloc: the HLLC step whose scratch is a static device array.

Some callers cannot allocate device memory -- a host whose own allocator owns all
of it, a framework recording a CUDA graph with its allocator frozen, a loop that
cannot take cudaMalloc's implicit synchronisation -- so this entry point keeps its
scratch in a fixed array inside the library instead of a caller workspace. This
test drives it through the C ABI with ctypes and checks two consecutive steps
against rb_hllc_step (the workspace entry point) on the same inputs: the states
must match bit for bit (the tolerance of every parity test in this suite) and the
banked loss to 1e-12 -- on a ragged grid with mixed edges, on a grid of exactly the
1,048,576-cell limit and on one-row and one-column strips of that length (the
largest ledger and stage-1 offsets the scratch holds). It also checks that a grid
above the limit is refused and that a non-finite state is reported through
rb_hllc_noalloc_read_error. The file is named to run last; it passes alone or after
the others.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _fields(ny, nx, dx, h, hu, hv, z, n, infil, bc):
    from rbsim import _lib

    P = ctypes.c_void_p
    f = _lib.HllcFields()
    f.ny, f.nx, f.dx = ny, nx, dx
    f.h = (P * 2)(h[0].data_ptr(), h[1].data_ptr())
    f.hu = (P * 2)(hu[0].data_ptr(), hu[1].data_ptr())
    f.hv = (P * 2)(hv[0].data_ptr(), hv[1].data_ptr())
    f.z, f.n = z.data_ptr(), n.data_ptr()
    f.h_comp, f.rain_field, f.infil = None, None, infil.data_ptr()
    f.bc[:] = bc
    return f


def _inputs(ny, nx, seed):
    rng = np.random.default_rng(seed)
    dev = torch.device("cuda")
    z = torch.from_numpy(rng.uniform(0.0, 0.5, (ny, nx)).astype(np.float32)).to(dev)
    h0 = torch.from_numpy(rng.uniform(0.2, 1.5, (ny, nx)).astype(np.float32)).to(dev)
    hu0 = torch.from_numpy(rng.uniform(-0.3, 0.3, (ny, nx)).astype(np.float32)).to(dev)
    hv0 = torch.from_numpy(rng.uniform(-0.3, 0.3, (ny, nx)).astype(np.float32)).to(dev)
    n = torch.full((ny, nx), 0.03, dtype=torch.float32, device=dev)
    infil = torch.full((ny, nx), 2e-6, dtype=torch.float32, device=dev)
    return z, h0, hu0, hv0, n, infil


def _pair(t):
    return [t.clone(), torch.zeros_like(t)]


def _read_noalloc_error():
    from rbsim import _lib

    err = ctypes.c_uint32(0)
    _lib.check(_lib.lib().rb_hllc_noalloc_read_error(ctypes.byref(err), torch.cuda.current_stream().cuda_stream))
    return err.value


@pytest.mark.parametrize("ny, nx, bc", [
    (300, 417, [0, 1, 2, 1]),     # ragged; north closed, south open, east fixed_stage, west open
    (1024, 1024, [1, 1, 1, 1]),   # exactly the cell limit, every edge open
    (1, 1 << 20, [1, 0, 2, 1]),   # one row of the limit's length
    (1 << 20, 1, [2, 1, 0, 0]),   # one column of it
])  # fmt: skip
def test_noalloc_step_matches_the_workspace_step_on_two_calls_in_a_row(ny, nx, bc):
    from rbsim import _lib

    L = _lib.lib()
    dx = 2.0
    z, h0, hu0, hv0, n, infil = _inputs(ny, nx, seed=21)
    stream = torch.cuda.current_stream().cuda_stream

    # reference run: rb_hllc_step with a caller-allocated workspace
    h, hu, hv = _pair(h0), _pair(hu0), _pair(hv0)
    fa = _fields(ny, nx, dx, h, hu, hv, z, n, infil, bc)
    nbytes = L.rb_hllc_workspace_bytes(ny, nx)
    ws = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    _lib.check(L.rb_workspace_init(ws.data_ptr(), nbytes, stream))

    # the same inputs through the no-allocation entry point
    g, gu, gv = _pair(h0), _pair(hu0), _pair(hv0)
    fb = _fields(ny, nx, dx, g, gu, gv, z, n, infil, bc)
    loss_b = torch.zeros(2, dtype=torch.float64, device="cuda")

    cur, banked_a = 0, []
    for k, dt in enumerate((0.05, 0.043)):
        args = _lib.StepArgs(dt, 0.0, 1.0, 0, 0, (ctypes.c_double * 4)(1.1, 1.2, 1.1, 1.3))
        _lib.check(L.rb_hllc_step(ctypes.byref(fa), cur, ctypes.byref(args), ws.data_ptr(), stream))
        out = ctypes.c_double()
        _lib.check(L.rb_ledger_loss(ws.data_ptr(), ny, nx, stream, ctypes.byref(out)))
        banked_a.append(out.value)
        rc = L.rb_hllc_step_noalloc(ctypes.byref(fb), cur, ctypes.byref(args),
                                    ctypes.c_void_p(loss_b.data_ptr() + 8 * k), stream)  # fmt: skip
        _lib.check(rc)
        cur ^= 1
        torch.cuda.synchronize()
        for a, b, name in ((h, g, "h"), (hu, gu, "hu"), (hv, gv, "hv")):
            np.testing.assert_array_equal(b[cur].cpu().numpy(), a[cur].cpu().numpy(), err_msg=f"call {k}: {name}")
    per_step_a = [banked_a[0], banked_a[1] - banked_a[0]]
    np.testing.assert_allclose(loss_b.cpu().numpy(), per_step_a, rtol=1e-12)
    assert abs(per_step_a[0]) > 0.0  # the edges really banked something
    assert _read_noalloc_error() == 0


def test_noalloc_step_reports_a_non_finite_state():
    """The HLLC stages clamp depth with max(h, 0), which turns a planted NaN into 0, so
    the non-finite state is made the way it can reach the stored depth: a uniform rain
    whose depth over the step overflows float32 (plain float arithmetic, no fault)."""
    from rbsim import _lib

    L = _lib.lib()
    ny, nx, dx = 64, 96, 1.0
    z, h0, hu0, hv0, n, infil = _inputs(ny, nx, seed=5)
    g, gu, gv = _pair(h0), _pair(hu0), _pair(hv0)
    f = _fields(ny, nx, dx, g, gu, gv, z, n, infil, [0, 0, 0, 0])
    args = _lib.StepArgs(10.0, 3.0e38, 1.0, 0, 0)
    stream = torch.cuda.current_stream().cuda_stream
    _lib.check(L.rb_hllc_step_noalloc(ctypes.byref(f), 0, ctypes.byref(args), None, stream))
    assert _read_noalloc_error() & _lib.RB_DEVERR_NONFINITE
    assert _read_noalloc_error() == 0  # read and cleared


def test_noalloc_step_refuses_grids_above_its_limit():
    from rbsim import _lib

    L = _lib.lib()
    ny, nx = 1025, 1024  # one row past 1,048,576 cells
    f = _lib.HllcFields()
    f.ny, f.nx, f.dx = ny, nx, 1.0
    args = _lib.StepArgs(0.01, 0.0, 1.0, 0, 0)
    rc = L.rb_hllc_step_noalloc(ctypes.byref(f), 0, ctypes.byref(args), None, None)
    assert rc == _lib.RB_ERR_ARG
    assert "1048576-cell" in _lib.last_error()
