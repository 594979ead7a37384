"""rbsim -- B200 solver hot path of river-basin-sim behind the reference's scheme API.

``get_scheme(name)`` returns the ``compute_dt`` / ``step`` module for
``"local_inertial"`` or ``"hllc_fv"``; ``State.from_bed`` builds the device state.
All solver arithmetic runs in librbsim.so (hand-written sm_100a CUDA).
"""

from .grid import GRAVITY, H_DRY, Grid
from .schemes import KNOWN_SCHEMES, get_scheme
from .state import State

__all__ = ["GRAVITY", "H_DRY", "Grid", "KNOWN_SCHEMES", "State", "get_scheme"]
