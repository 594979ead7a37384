"""Staggered uniform-raster geometry (the layout of solver/core/grid.py:1-86).

Cells ``(ny, nx)`` carry ``h``, ``z``, ``eta = h + z``; x-faces ``(ny, nx+1)`` carry
``qx`` with ``qx[i, j]`` between cells ``(i, j-1)`` and ``(i, j)``; y-faces
``(ny+1, nx)`` carry ``qy`` with ``qy[i, j]`` between ``(i-1, j)`` and ``(i, j)``.
Positive ``qx`` flows +x (increasing column), positive ``qy`` flows +y (increasing
row). Row-major float32 throughout.
"""

from __future__ import annotations

from dataclasses import dataclass

GRAVITY = 9.81  # grid.py:43
H_DRY = 1.0e-3  # grid.py:48


@dataclass(frozen=True)
class Grid:
    ny: int
    nx: int
    dx: float

    @property
    def shape(self) -> tuple[int, int]:
        return (self.ny, self.nx)

    @property
    def qx_shape(self) -> tuple[int, int]:
        return (self.ny, self.nx + 1)

    @property
    def qy_shape(self) -> tuple[int, int]:
        return (self.ny + 1, self.nx)

    @property
    def cell_area(self) -> float:
        return self.dx * self.dx

    @property
    def n_cells(self) -> int:
        return self.ny * self.nx
