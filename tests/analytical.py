"""Closed-form 1-D dam-break solutions on a flat frictionless bed (dam at x = 0).

The validation references the reference's dam-break gates are written against
(validation/analytical.py there; test_dam_break.py:94, :143): Stoker's wet-bed
solution (rarefaction, constant star state, bore) and Ritter's dry-bed
rarefaction. Standard shallow-water results, written here from the Riemann
problem: the star depth h_m solves 2(sqrt(g h_l) - sqrt(g h_m)) =
(h_m - h_r) sqrt(g (h_m + h_r) / (2 h_m h_r)); the bore moves at
s = h_m u_m / (h_m - h_r).
"""

from __future__ import annotations

import math

import numpy as np

G = 9.81


def star_depth(h_l: float, h_r: float, g: float = G) -> float:
    def mismatch(h):
        return 2.0 * (math.sqrt(g * h_l) - math.sqrt(g * h)) - (h - h_r) * math.sqrt(0.5 * g * (h + h_r) / (h * h_r))

    lo, hi = h_r, h_l
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if mismatch(mid) > 0.0:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def stoker(x, t: float, h_l: float, h_r: float, g: float = G):
    x = np.asarray(x, dtype=np.float64)
    c_l = math.sqrt(g * h_l)
    h_m = star_depth(h_l, h_r, g)
    c_m = math.sqrt(g * h_m)
    u_m = 2.0 * (c_l - c_m)
    s = h_m * u_m / (h_m - h_r)
    xi = x / t
    h = np.where(xi <= -c_l, h_l, 0.0)
    fan = (xi > -c_l) & (xi < u_m - c_m)
    h = np.where(fan, ((2.0 * c_l - xi) / 3.0) ** 2 / g, h)
    h = np.where((xi >= u_m - c_m) & (xi < s), h_m, h)
    h = np.where(xi >= s, h_r, h)
    return h


def stoker_front(t: float, h_l: float, h_r: float, g: float = G) -> float:
    h_m = star_depth(h_l, h_r, g)
    u_m = 2.0 * (math.sqrt(g * h_l) - math.sqrt(g * h_m))
    return h_m * u_m / (h_m - h_r) * t


def ritter(x, t: float, h_l: float, g: float = G):
    x = np.asarray(x, dtype=np.float64)
    c_l = math.sqrt(g * h_l)
    xi = x / t
    h = np.where(xi <= -c_l, h_l, 0.0)
    fan = (xi > -c_l) & (xi < 2.0 * c_l)
    return np.where(fan, (2.0 * c_l - xi) ** 2 / (9.0 * g), h)
