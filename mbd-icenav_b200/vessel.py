"""3-DOF supply-vessel constants (host side, computed once).

Restates the Fossen bis-scaled supply-vessel model the reference takes from
AUTO-IceNav (``medea_ice_ship/auto_icenav_ship.py:100-173``) and the ship
hull / controller-gain construction of ``build_ship_dynamics_data``
(``medea_ice_ship/jax_ice_state.py:270-343``).  The numbers in ``_MBIS``,
``_DBIS``, ``_THRUST_K`` and ``_THRUSTER_CFG`` are the published model
constants of that vessel (Fossen 2021 supply model); they must be identical
for the dynamics to be the same.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .config import DEFAULT_MATERIAL

_G = 9.81
_MBIS = np.array([[1.1274, 0.0, 0.0], [0.0, 1.8902, -0.0744], [0.0, -0.0744, 0.1278]])
_DBIS = np.array([[0.0358, 0.0, 0.0], [0.0, 0.1183, -0.0124], [0.0, -0.0041, 0.0308]])
_THRUST_K = np.array([3.2, 3.2, 3.2, 3.2, 31.2, 31.2])
_THRUSTER_CFG = np.array([[0, 0, 0, 0, 1, 1],
                          [1, 1, 1, 1, 0, 0],
                          [30, 22, -22, -30, -8, 8]], dtype=float)
_N_MAX = np.array([250.0, 250.0, 250.0, 250.0, 160.0, 160.0])


@dataclass
class SupplyVessel:
    """Mass, damping and thruster matrices of the bis-scaled supply vessel."""

    mass: float = 6000.0e3
    length: float = 76.2

    def __post_init__(self):
        scale = np.diag([1.0, 1.0, self.length])
        self.T_n = 1.0
        self.n_max = _N_MAX.copy()
        self.B = _THRUSTER_CFG @ np.diag(_THRUST_K)
        self.M3 = self.mass * (scale @ _MBIS @ scale)
        self.M3inv = np.linalg.inv(self.M3)
        self.D3 = self.mass * math.sqrt(_G / self.length) * (scale @ _DBIS @ scale)
        self.wn = np.diag([0.1, 0.1, 0.2])
        self.zeta = np.diag([1.0 / math.sqrt(2.0)] * 3)


@dataclass
class ShipProperties:
    """Ship principal dimensions and displacement mass (``properties.py:25-38``)."""

    length: float
    beam: float
    draft: float
    displacement: float = None

    def __post_init__(self):
        if self.displacement is None:
            self.displacement = (self.length * self.beam * self.draft * 0.6
                                 * DEFAULT_MATERIAL.water_density)
        self.mass = self.displacement


def tapered_hull_outline(ship_length: float, ship_beam: float, n_pts: int = 30) -> np.ndarray:
    """Closed hull outline in the body frame, bow at +x: (2*(n_pts+1), 2).

    Starboard side from bow to stern, then port side from stern to bow; the
    half-beam tapers as ``1 - 0.9*((x/L2 - 0.6)/0.4)^1.5`` ahead of 60 % of
    the half-length, floored at 2 % (``jax_ice_state.py:305-328``).
    """
    half_len = ship_length / 2.0
    half_beam = ship_beam / 2.0

    def half_width(x_loc):
        x_rel = x_loc / half_len
        taper = 1.0 - 0.9 * ((x_rel - 0.6) / 0.4) ** 1.5 if x_rel > 0.6 else 1.0
        return half_beam * max(taper, 0.02)

    xs = [half_len - (i / n_pts) * ship_length for i in range(n_pts + 1)]
    starboard = [(x, half_width(x)) for x in xs]
    port = [(x, -half_width(x)) for x in reversed(xs)]
    return np.array(starboard + port, dtype=np.float64)


def pointed_hull_outline(ship_length: float, ship_beam: float) -> np.ndarray:
    """A 7-vertex pointed hull (bow at +x), 60 x 12 m in the seeded benchmark fields."""
    L2, B2 = ship_length / 2.0, ship_beam / 2.0
    return np.array([[L2, 0.0], [0.5 * L2, B2], [-0.8 * L2, B2], [-L2, 0.6 * B2],
                     [-L2, -0.6 * B2], [-0.8 * L2, -B2], [0.5 * L2, -B2]], dtype=np.float64)
