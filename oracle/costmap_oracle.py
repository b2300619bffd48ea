"""NumPy restatement of the reference's KE costmap (test infrastructure only).

Follows ``medea_ice_ship/jax_costmap.py`` as the reference runs it in its
tests (float64 mode, ``test_jax_costmap.py:23``): the per-element KE constant
is computed in float64 and clipped to float32 (``:256-268``); the rasteriser
works on float32 arrays, with its float arguments (origin, resolution, buffer
factor) entering as weak scalars, i.e. rounded to float32 where they meet the
float32 arrays (``:99-139``); the open-water floor is a float32 maximum
(``:286``); the SIC modulation (``:271-284``) is a float64 box mean of the
ice-covered cells as SciPy's ``uniform_filter`` accumulates it, then a
float32 power; the ship-footprint dilation is a square max window over an
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


def sic_window(rows: int, cols: int) -> int:
    """Box size of the SIC estimate: odd, at most 31 cells (jax_costmap.py:274-276)."""
    k = min(31, (min(rows, cols) // 4) | 1)
    return k + 1 if k % 2 == 0 else k


def box_mean_1d(line: np.ndarray, size: int) -> np.ndarray:
    """Mean over a centred window of ``size`` (``size // 2`` before, the rest
    after) with mirror padding at the ends (d c b a | a b c d | d c b a), as a
    running sum in float64: the first window summed in order, then each step
    adds (entering - leaving).  This is the order in which SciPy's
    ``uniform_filter1d`` accumulates (checked bit for bit against it)."""
    s1 = size // 2
    s2 = size - s1 - 1
    ext = np.pad(np.asarray(line, np.float64), (s1, s2), mode="symmetric")
    out = np.empty(len(line), np.float64)
    tmp = 0.0
    for k in range(size):
        tmp += ext[k]
    out[0] = tmp / size
    for i in range(1, len(line)):
        tmp += ext[i + size - 1] - ext[i - 1]
        out[i] = tmp / size
    return out


def sic_modulate(grid: np.ndarray, weight: float) -> np.ndarray:
    """grid * SIC^weight, SIC the local fraction of ice-covered cells
    (jax_costmap.py:271-284): a box mean of (grid > 0) along axis 0, then
    axis 1 (scipy.ndimage.uniform_filter, mode "reflect"), clipped to [0, 1],
    float32, floored at 1e-6, raised to ``weight`` in float32."""
    rows, cols = grid.shape
    k = sic_window(rows, cols)
    occ = (grid > 0.0).astype(np.float64)
    a = np.stack([box_mean_1d(occ[:, c], k) for c in range(cols)], 1)
    sic = np.stack([box_mean_1d(a[r, :], k) for r in range(rows)], 0)
    sic = np.clip(sic, 0.0, 1.0).astype(np.float32)
    sic_safe = np.maximum(sic, 1e-6)
    return grid * np.power(sic_safe, weight)


def build_costmap(centroids, thicknesses, radii, x_min, x_max, y_min, y_max, *, resolution=2.0, margin=20.0,
                  base_cost=0.1, collision_cost=5.0, obs_cost_buffer_factor=0.1, ship_length=None,
                  ship_beam=None, planning_clearance_margin=0.0, ship_speed=4.0, ship_mass=23e6,
                  ke_cost_scale=1e-6, masses=None, ice_resistance_weight=0.0):
    """``build_costmap_jax`` (jax_costmap.py:179-331); returns (grid, geometry)."""
    x0, y0, width, height, rows, cols = grid_geometry(x_min, x_max, y_min, y_max, resolution, margin)
    n = len(centroids)
    if n > 0:
        if masses is None:
            masses = math.pi * np.asarray(radii, np.float64) ** 2 * np.asarray(thicknesses, np.float64) \
                * ICE_DENSITY_APPROX
        kw = ke_constants(masses, collision_cost, ship_speed, ship_mass, ke_cost_scale)
        grid = rasterize(centroids, radii, kw, x0, y0, resolution, rows, cols, obs_cost_buffer_factor)
        if ice_resistance_weight > 0.0:
            grid = sic_modulate(grid, ice_resistance_weight)
        grid = np.maximum(grid, np.float32(base_cost))
    else:
        grid = np.full((rows, cols), float(base_cost), np.float32)
    if ship_length is not None and ship_beam is not None and ship_length > 0 and ship_beam > 0:
        grid = dilate(grid, dilation_half(ship_beam, planning_clearance_margin, resolution))
    return grid, dict(x_origin=x0, y_origin=y0, width=width, height=height, rows=rows, cols=cols)
