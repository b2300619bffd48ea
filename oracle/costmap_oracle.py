"""NumPy restatement of the reference's KE costmap (test infrastructure only).

Follows ``medea_ice_ship/jax_costmap.py`` as the reference runs it in its
tests (float64 mode, ``test_jax_costmap.py:23``): the per-element KE constant
is computed in float64 and clipped to float32 (``:256-268``); the rasteriser
works on float32 arrays, with its float arguments (origin, resolution, buffer
factor) entering as weak scalars, i.e. rounded to float32 where they meet the
float32 arrays (``:99-139``); the open-water floor is a float32 maximum
(``:286``); the ship-footprint dilation is a square max window over an
edge-padded grid (``:87-95``, ``:142-176``, ``:292-298``).  Pinned by
``tests/test_costmap.py`` against ``tests/golden/costmap_golden.npz``.
"""
from __future__ import annotations

import math

import numpy as np

ICE_DENSITY_APPROX = 920.0  # jax_costmap.py:259 (mass when none is given)


def grid_geometry(x_min, x_max, y_min, y_max, resolution, margin):
    """(x_origin, y_origin, width, height, rows, cols) (jax_costmap.py:237-244)."""
    x_origin = x_min - margin
    y_origin = y_min - margin
    width = (x_max - x_min) + 2.0 * margin
    height = (y_max - y_min) + 2.0 * margin
    cols = max(1, int(np.ceil(width / resolution)))
    rows = max(1, int(np.ceil(height / resolution)))
    return x_origin, y_origin, width, height, rows, cols


def ke_constants(masses, collision_cost, ship_speed, ship_mass, ke_cost_scale) -> np.ndarray:
    """Per-element KE cost constant, float64 then clipped to float32 (jax_costmap.py:261-268)."""
    v = max(float(ship_speed), 1e-6)
    M_s = float(ship_mass)
    m_i = np.asarray(masses, np.float64)
    ke = (float(collision_cost) * v * v * m_i * M_s * (m_i + 2.0 * M_s) / (2.0 * (M_s + m_i) ** 2)
          * float(ke_cost_scale))
    return np.clip(ke, 0.0, 1e8).astype(np.float32)


def rasterize(centroids, radii, ke_w, x_origin, y_origin, resolution, rows, cols, buffer_factor) -> np.ndarray:
    """Max over elements of ke * max(0, (eff_r^2 - d^2) / eff_r^2) (jax_costmap.py:99-139)."""
    f = np.float32
    c = np.asarray(centroids, np.float64).astype(f).reshape(-1, 2)
    r = np.asarray(radii, np.float64).astype(f)
    w = np.asarray(ke_w, f)
    cell_x = f(x_origin) + (np.arange(cols, dtype=f) + f(0.5)) * f(resolution)
    cell_y = f(y_origin) + (np.arange(rows, dtype=f) + f(0.5)) * f(resolution)
    XX, YY = np.meshgrid(cell_x, cell_y)
    grid = np.zeros((rows, cols), f)
    buf = f(1.0 + buffer_factor)
    half = f(0.5 * resolution)
    for i in range(len(r)):
        eff = r[i] * buf + half
        dsq = (XX - c[i, 0]) ** 2 + (YY - c[i, 1]) ** 2
        fall = np.maximum(f(0.0), (eff ** 2 - dsq) / (eff ** 2))
        grid = np.maximum(grid, w[i] * fall)
    return grid.astype(f)


def dilation_half(ship_beam, planning_clearance_margin, resolution) -> int:
    """Half width of the square max window (0: no dilation) (jax_costmap.py:87-95, :292-298)."""
    if ship_beam is None or not ship_beam > 0:
        return 0
    inflation_r = 0.5 * ship_beam + planning_clearance_margin
    if not inflation_r > 0:
        return 0
    return int(np.ceil(inflation_r / resolution))


def dilate(grid, half: int) -> np.ndarray:
    """Max over a (2 half + 1)^2 window of the edge-padded grid (jax_costmap.py:142-176)."""
    if half <= 0:
        return grid
    p = np.pad(grid, ((half, half), (half, half)), mode="edge")
    k = 2 * half + 1
    win = np.lib.stride_tricks.sliding_window_view(p, (k, k))
    return np.maximum(win.max(axis=(2, 3)), np.float32(-np.inf)).astype(np.float32)


def build_costmap(centroids, thicknesses, radii, x_min, x_max, y_min, y_max, *, resolution=2.0, margin=20.0,
                  base_cost=0.1, collision_cost=5.0, obs_cost_buffer_factor=0.1, ship_length=None,
                  ship_beam=None, planning_clearance_margin=0.0, ship_speed=4.0, ship_mass=23e6,
                  ke_cost_scale=1e-6, masses=None):
    """``build_costmap_jax`` without SIC modulation (jax_costmap.py:179-331); returns (grid, geometry)."""
    x0, y0, width, height, rows, cols = grid_geometry(x_min, x_max, y_min, y_max, resolution, margin)
    n = len(centroids)
    if n > 0:
        if masses is None:
            masses = math.pi * np.asarray(radii, np.float64) ** 2 * np.asarray(thicknesses, np.float64) \
                * ICE_DENSITY_APPROX
        kw = ke_constants(masses, collision_cost, ship_speed, ship_mass, ke_cost_scale)
        grid = rasterize(centroids, radii, kw, x0, y0, resolution, rows, cols, obs_cost_buffer_factor)
        grid = np.maximum(grid, np.float32(base_cost))
    else:
        grid = np.full((rows, cols), float(base_cost), np.float32)
    if ship_length is not None and ship_beam is not None and ship_length > 0 and ship_beam > 0:
        grid = dilate(grid, dilation_half(ship_beam, planning_clearance_margin, resolution))
    return grid, dict(x_origin=x0, y_origin=y0, width=width, height=height, rows=rows, cols=cols)
