"""Reservoir host logic without a device: barriers, structure rules, the pool gauge.

These restate solver/processes/test_reservoir.py:91, :297, :303, :313 and the
structure checks of solver/io/test_config.py:241-305. The release transfer itself
(``rb_reservoir_withdraw`` / ``rb_reservoir_deliver``) is a device call, gated in
tests/gates.py on both backends. Everything here runs before it or without it. A
stand-in state with CPU tensors for ``h`` and ``z`` drives the operator's gauge and
its dry-pool path.
"""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import pytest
import torch

from rbsim.config import Structure
from rbsim.grid import H_DRY, Grid
from rbsim.processes.reservoir import ReservoirOperator, apply_barriers, build_operators

NY, NX = 6, 8


def _dam(**kw):
    base = dict(name="dam", cells=[(3, c) for c in range(NX)], crest_m=5.0, release_rule="fixed",
                release_m3_s=2.0, pool=(0, 0, 2, NX - 1), outlet=(5, 3, 5, 3))  # fmt: skip
    base.update(kw)
    return Structure(**base)


def _stand_in(z, h):
    return SimpleNamespace(grid=Grid(ny=z.shape[0], nx=z.shape[1], dx=10.0), device=torch.device("cpu"),
                           z=torch.from_numpy(np.asarray(z, np.float32)),
                           h=torch.from_numpy(np.asarray(h, np.float32)), arm_loss_accumulator=lambda: None)  # fmt: skip


def test_apply_barriers_raises_the_bed_and_never_lowers_it():
    """test_reservoir.py:91."""
    bed = np.zeros((5, 5), np.float32)
    bed[2, 2] = 7.0
    out = apply_barriers(bed, [Structure(name="d", cells=[(2, 2), (2, 3)], crest_m=4.0)])
    assert out[2, 3] == 4.0 and out[2, 2] == 7.0 and bed[2, 3] == 0.0
    assert apply_barriers(bed, []) is bed
    with pytest.raises(ValueError, match="outside"):
        apply_barriers(bed, [Structure(name="d", cells=[(9, 9)], crest_m=1.0)])


@pytest.mark.parametrize("kw, needle", [
    (dict(kind="weir"), "type must be"),
    (dict(cells=[]), "at least one barrier cell"),
    (dict(release_rule="sometimes"), "release_rule must be"),
    (dict(kind="levee"), "levee is barrier geometry only"),
    (dict(interval_s=0.0), "interval_s must be > 0"),
    (dict(pool=None), "needs both a 'pool' box and an 'outlet'"),
    (dict(pool=(2, 0, 0, 3)), "pool must be"),
    (dict(outlet=(5, 4, 5, 3)), "outlet must be"),
    (dict(outlet=(1, 1, 1, 1)), "overlaps the pool"),
    (dict(release_m3_s=0.0), "needs release_m3_s > 0"),
    (dict(release_rule="target_stage", target_stage_m=None, release_max_m3_s=3.0), "needs target_stage_m"),
    (dict(release_rule="target_stage", target_stage_m=3.0, release_max_m3_s=0.0), "needs release_max_m3_s > 0"),
    (dict(release_rule="target_stage", target_stage_m=6.0, release_max_m3_s=3.0), "must be below crest_m"),
])  # fmt: skip
def test_a_structure_that_cannot_be_operated_is_refused(kw, needle):
    """solver/io/test_config.py:305: each refusal names what is wrong."""
    with pytest.raises(ValueError, match=needle):
        _dam(**kw)


def test_release_rules():
    """Open-loop ``fixed``; ``target_stage`` ramps from 0 at the target to the cap at the crest."""
    fixed = _dam()
    assert fixed.discharge_at(1.0) == 2.0 and fixed.discharge_at(None) == 0.0
    ramp = _dam(release_rule="target_stage", target_stage_m=3.0, release_max_m3_s=8.0)
    assert ramp.discharge_at(2.0) == 0.0 and ramp.discharge_at(3.0) == 0.0
    assert ramp.discharge_at(4.0) == pytest.approx(4.0) and ramp.discharge_at(9.0) == 8.0
    assert Structure(name="l", kind="levee", cells=[(0, 0)], crest_m=1.0).discharge_at(5.0) == 0.0


def test_build_operators_skips_structures_without_a_rule():
    """test_reservoir.py:297."""
    st = _stand_in(np.zeros((NY, NX)), np.zeros((NY, NX)))
    ops = build_operators([_dam(name="barrier", release_rule="none"), _dam(name="live")], st)
    assert [o.structure.name for o in ops] == ["live"]


def test_operator_rejects_boxes_outside_the_grid():
    """test_reservoir.py:303, and the same for the outlet."""
    st = _stand_in(np.zeros((NY, NX)), np.zeros((NY, NX)))
    with pytest.raises(ValueError, match="outside the"):
        ReservoirOperator(_dam(pool=(0, 0, 2, NX + 40)), st)
    with pytest.raises(ValueError, match="outside the"):
        ReservoirOperator(_dam(outlet=(NY + 1, 0, NY + 1, 0)), st)
    with pytest.raises(ValueError, match="no release rule"):
        ReservoirOperator(_dam(release_rule="none"), st)


def test_pool_stage_gauges_the_deepest_cell_not_the_highest_water():
    """test_reservoir.py:313: a film high on the pool's wall does not read as the stage."""
    z = np.full((NY, NX), 4.0, np.float32)
    z[1, 5] = 1.0  # the deepest bed cell of the pool box is the gauge
    h = np.zeros((NY, NX), np.float32)
    h[0, 0] = 0.5  # a film on a high cell: z + h = 4.5, above the true pool level
    h[1, 5] = 2.0  # the pool: z + h = 3.0
    op = ReservoirOperator(_dam(), _stand_in(z, h))
    assert op.pool_stage() == pytest.approx(3.0)
    h[1, 5] = 0.5 * H_DRY
    assert ReservoirOperator(_dam(), _stand_in(z, h)).pool_stage() is None


def test_a_release_from_a_dry_pool_moves_nothing():
    """test_reservoir.py:191, on the host path: a dry gauge asks for no release, so no transfer runs."""
    z = np.full((NY, NX), 4.0, np.float32)
    op = ReservoirOperator(_dam(release_rule="target_stage", target_stage_m=3.0, release_max_m3_s=8.0),
                           _stand_in(z, np.zeros((NY, NX))))  # fmt: skip
    rec = op.advance(900.0, 900.0)
    assert rec.stage is None and rec.discharge_m3_s == 0.0 and rec.volume_m3 == 0.0
    assert op.series == [{"time": 900.0, "stage": None, "discharge_m3_s": 0.0, "volume_m3": 0.0}]
