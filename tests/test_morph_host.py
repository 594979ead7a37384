"""Host-side refusals and bounds of the morphology API, without a device.

These restate the reference's argument tests for ``bed_change_bounds``,
``arm_sediment`` and ``MorphologyProcess`` (solver/processes/test_morphology.py:236,
:302, :318; solver/core/test_sediment.py:705, :714, :772, :780, :787). Every refusal
here is raised before anything is allocated on a device. So a stand-in state that
carries only a grid, a ``sediment`` slot and the CPU device exercises the same code a
CUDA state does. A refused arming must leave the state unarmed.
"""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import pytest
import torch

from rbsim.grid import Grid
from rbsim.processes.morphology import MorphologyProcess, bed_change_bounds
from rbsim.sediment import SedimentError, arm_sediment, validate_grain_size


def _stand_in(ny=3, nx=4, armed=False):
    sed = SimpleNamespace(porosity=0.4) if armed else None
    return SimpleNamespace(grid=Grid(ny=ny, nx=nx, dx=5.0), sediment=sed, device=torch.device("cpu"))


def test_bed_change_bounds_are_unbounded_until_something_asks_for_a_limit():
    """solver/processes/test_morphology.py:236."""
    lo, hi = bed_change_bounds((3, 4))
    assert (lo == -np.inf).all() and (hi == np.inf).all()
    lo, hi = bed_change_bounds((3, 4), alluvium_thickness=0.25)
    assert (lo == np.float32(-0.25)).all() and (hi == np.inf).all()
    thick = np.full((3, 4), 0.5, np.float32)
    thick[1, 1] = 0.0
    lo, hi = bed_change_bounds((3, 4), alluvium_thickness=thick, frozen_cells=[(0, 0)])
    assert lo[1, 1] == 0.0 and hi[1, 1] == np.inf
    assert lo[0, 0] == 0.0 and hi[0, 0] == 0.0
    assert lo.dtype == hi.dtype == np.float32
    with pytest.raises(SedimentError, match="outside"):
        bed_change_bounds((3, 4), frozen_cells=[(9, 9)])
    with pytest.raises(SedimentError, match=">= 0"):
        bed_change_bounds((3, 4), alluvium_thickness=-1.0)
    with pytest.raises(SedimentError, match="shape"):
        bed_change_bounds((3, 4), alluvium_thickness=np.zeros((2, 2), np.float32))


def test_a_scalar_grain_size_broadcasts_to_a_bit_exact_uniform_field():
    """solver/core/test_sediment.py:705."""
    grain = validate_grain_size(0.0123, Grid(ny=3, nx=4, dx=5.0))
    assert grain.dtype == np.float32 and (grain == np.float32(0.0123)).all()


def test_a_grain_size_field_is_carried_per_cell():
    """solver/core/test_sediment.py:714 (the field part; zeros are allowed)."""
    field = np.full((3, 4), 0.004, np.float32)
    field[1, 2] = 0.0
    field[0, 0] = 0.016
    grain = validate_grain_size(field, Grid(ny=3, nx=4, dx=5.0))
    assert (grain == field).all() and grain is not field


@pytest.mark.parametrize(
    "bad, match",
    [(np.zeros((2, 2), np.float32), "shape"), (np.full((3, 4), -1.0, np.float32), ">= 0"),
     (np.full((3, 4), np.nan, np.float32), "non-finite")],
)  # fmt: skip
def test_a_grain_size_that_cannot_mean_anything_is_refused(bad, match):
    """solver/core/test_sediment.py:772."""
    st = _stand_in()
    with pytest.raises(SedimentError, match=match):
        arm_sediment(st, bad, 0.4)
    assert st.sediment is None


@pytest.mark.parametrize("p", [0.0, 1.0, 1.5, -0.1])
def test_a_porosity_exner_cannot_divide_by_is_refused(p):
    """solver/core/test_sediment.py:780."""
    st = _stand_in()
    with pytest.raises(SedimentError, match="porosity"):
        arm_sediment(st, 0.008, p)
    assert st.sediment is None


def test_arming_twice_is_refused_rather_than_silently_resetting_the_ledger():
    """solver/core/test_sediment.py:787."""
    with pytest.raises(SedimentError, match="already armed"):
        arm_sediment(_stand_in(armed=True), 0.008, 0.4)


def test_the_process_refuses_what_it_cannot_honour():
    """solver/processes/test_morphology.py:302."""
    with pytest.raises(SedimentError, match="arm_sediment"):
        MorphologyProcess(_stand_in(), interval_s=60.0)
    st = _stand_in(armed=True)
    with pytest.raises(SedimentError, match="interval_s"):
        MorphologyProcess(st, interval_s=0.0)
    lo, hi = bed_change_bounds(st.grid.shape)
    with pytest.raises(SedimentError, match="both"):
        MorphologyProcess(st, interval_s=60.0, dz_lo=lo)
    with pytest.raises(SedimentError, match="grid"):
        MorphologyProcess(st, interval_s=60.0, dz_lo=lo[:2], dz_hi=hi[:2])
    with pytest.raises(SedimentError, match="cross"):
        MorphologyProcess(st, interval_s=60.0, dz_lo=hi, dz_hi=lo)


def test_the_process_counts_frozen_and_floored_cells():
    """What ``summary`` and the store's attributes report about the bounds."""
    st = _stand_in(armed=True)
    lo, hi = bed_change_bounds(st.grid.shape, alluvium_thickness=0.1, frozen_cells=[(0, 0), (2, 3)])
    morph = MorphologyProcess(st, interval_s=60.0, dz_lo=lo, dz_hi=hi)
    assert morph.frozen_cells == 2 and morph.floored_cells == 10


def test_an_activation_covering_more_than_its_interval_is_refused():
    """solver/processes/test_morphology.py:318: refused before the bed is touched."""
    morph = MorphologyProcess(_stand_in(armed=True), interval_s=60.0)
    with pytest.raises(SedimentError, match="collapsed"):
        morph.advance(180.0, 180.0)
    assert morph.records == []
