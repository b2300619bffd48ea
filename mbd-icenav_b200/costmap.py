"""KE collision costmap on the GPU — drop-in for ``medea_ice_ship.jax_costmap``.

``build_costmap_jax`` and ``build_costmap_jax_from_ice_state`` keep the
reference's signatures and defaults (``jax_costmap.py:179-357``) and return the
same ``JaxCostMapResult`` (``:31-79``).  The grid is built by ``dem_ke_costmap``
(``csrc/dem_costmap.cu``) and equals the reference's float32 grid bit for bit.
Inputs may be NumPy arrays, torch tensors or anything exposing ``__dlpack__``
(a JAX array, a live ``IceState`` field); ``result.grid`` keeps the grid on the
device, and ``download=False`` skips the copy into ``result.cost_map``.

The SIC modulation (``ice_resistance_weight > 0``, ``:271-284``), which the
reference runs on the host with SciPy's box filter, runs on the device in the
same float64 operation order.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import Any, Optional, Tuple

import numpy as np

from . import _abi


@dataclass
class JaxCostMapResult:
    """The reference's costmap result (``jax_costmap.py:31-79``) plus the device grid."""

    cost_map: Any
    x_origin: float
    y_origin: float
    resolution: float
    rows: int
    cols: int
    width: float
    height: float
    base_cost: float = 0.1
    grid: Any = None  # (rows, cols) float32 torch tensor on the device

    def get_cost_world(self, x: float, y: float) -> float:
        """Cell value at world (x, y), or ``base_cost`` outside the grid (``jax_costmap.py:71-79``)."""
        col = int((x - self.x_origin) / self.resolution)
        row = int((y - self.y_origin) / self.resolution)
        if 0 <= row < self.rows and 0 <= col < self.cols:
            return float(self.cost_map[row, col])
        return float(self.base_cost)


def _tensor(x, device):
    import torch
    if isinstance(x, torch.Tensor):
        t = x
    elif hasattr(x, "__dlpack__") and not isinstance(x, np.ndarray):
        t = torch.from_dlpack(x)
    else:
        t = torch.as_tensor(np.asarray(x, dtype=np.float64))
    if t.dtype not in (torch.float32, torch.float64):
        t = t.to(torch.float64)
    return t.to(device).contiguous()


def build_costmap_jax(centroids, thicknesses, radii, x_min: float, x_max: float, y_min: float, y_max: float, *,
                      resolution: float = 2.0, margin: float = 20.0, base_cost: float = 0.1,
                      collision_cost: float = 5.0, obs_cost_buffer_factor: float = 0.1,
                      ship_length: Optional[float] = None, ship_beam: Optional[float] = None,
                      planning_clearance_margin: float = 0.0, verbose: bool = False, ship_speed: float = 4.0,
                      ship_mass: float = 23e6, ke_cost_scale: float = 1e-6, ice_resistance_weight: float = 0.0,
                      masses=None, device=None, download: bool = True) -> Tuple[JaxCostMapResult, dict]:
    """KE collision costmap of the ice elements (``jax_costmap.py:179-331``)."""
    import torch
    if not ice_resistance_weight >= 0.0:
        raise ValueError("ice_resistance_weight must be >= 0")
    lib = _abi.load_library()
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    # grid geometry in double, as the reference (jax_costmap.py:237-244)
    x_origin = x_min - margin
    y_origin = y_min - margin
    width = (x_max - x_min) + 2.0 * margin
    height = (y_max - y_min) + 2.0 * margin
    cols = max(1, int(np.ceil(width / resolution)))
    rows = max(1, int(np.ceil(height / resolution)))
    if verbose:
        print(f"  [jax-costmap] grid: {rows}×{cols} cells ({rows * cols / 1e6:.2f} M), n_elem={len(radii)}",
              flush=True)
    cents = _tensor(centroids, dev).reshape(-1, 2)
    n = int(cents.shape[0])
    dt = cents.dtype
    rad = _tensor(radii, dev).to(dt)
    thick = _tensor(thicknesses, dev).to(dt) if masses is None else None
    mass = _tensor(masses, dev).to(dt) if masses is not None else None
    half = 0
    if ship_length is not None and ship_beam is not None and ship_length > 0 and ship_beam > 0:
        inflation_r = 0.5 * ship_beam + planning_clearance_margin
        if inflation_r > 0:
            half = int(math.ceil(inflation_r / resolution))  # jax_costmap.py:87-95
    P = _abi.DemCostmapParams(x_origin=x_origin, y_origin=y_origin, resolution=resolution, rows=rows, cols=cols,
                              base_cost=base_cost, collision_cost=collision_cost,
                              obs_cost_buffer_factor=obs_cost_buffer_factor, ship_speed=ship_speed,
                              ship_mass=ship_mass, ke_cost_scale=ke_cost_scale, dilate_half=half,
                              has_masses=1 if masses is not None else 0,
                              ice_resistance_weight=float(ice_resistance_weight))
    sic = None
    if ice_resistance_weight > 0.0:
        sic = torch.empty(rows * cols, dtype=torch.float64, device=dev)
        P.sic_scratch = sic.data_ptr()
    grid = torch.empty((rows, cols), dtype=torch.float32, device=dev)
    tmp = torch.empty((rows, cols), dtype=torch.float32, device=dev) if half > 0 else None
    flag = torch.empty(1, dtype=torch.int32, device=dev)
    ptr = lambda t: None if t is None else t.data_ptr()
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    code = _abi.DEM_F32 if dt == torch.float32 else _abi.DEM_F64
    rc = lib.dem_ke_costmap(code, n, ptr(cents) if n else None, ptr(rad) if n else None,
                            ptr(thick) if n else None, ptr(mass) if n else None, C.byref(P), grid.data_ptr(),
                            ptr(tmp), flag.data_ptr(), stream)
    if rc != _abi.DEM_OK:
        raise _abi.DemError(rc, "dem_ke_costmap failed")
    cost_map = grid.cpu().numpy() if download else None
    result = JaxCostMapResult(cost_map=cost_map, x_origin=float(x_origin), y_origin=float(y_origin),
                              resolution=float(resolution), rows=int(rows), cols=int(cols), width=float(width),
                              height=float(height), base_cost=float(base_cost), grid=grid)
    bounds = {"x_min": float(x_min), "x_max": float(x_max), "y_min": float(y_min), "y_max": float(y_max),
              "x_origin": float(x_origin), "y_origin": float(y_origin), "width": float(width),
              "height": float(height)}
    return result, bounds


def build_costmap_jax_from_ice_state(state, static, x_min: float, x_max: float, y_min: float, y_max: float,
                                     **kwargs) -> Tuple[JaxCostMapResult, dict]:
    """Costmap of a live ``IceState`` with its ``IceStaticData`` masses (``jax_costmap.py:334-357``)."""
    return build_costmap_jax(state.positions, static.thicknesses, static.radii, x_min, x_max, y_min, y_max,
                             masses=static.masses, **kwargs)
