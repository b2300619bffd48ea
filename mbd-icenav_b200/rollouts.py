"""Batched planner rollouts through the DEM (one persistent launch per batch).

A sampling planner scores many candidate control sequences for the ship.
Here each candidate is one system of a multi-system ``FrameStep``: its own
copy of the ice in a local window cut along its predicted path (uneven
sizes), its own ship driven by its controls through ``dem_rollout_segment``
(the frame step with ``tau = u + tau_ice``), all H steps of all candidates in
one launch.  ``costs`` then scores every candidate on the device
(``dem_rollout_costs``): the reference planner's four raw cost components
(``jax_mbd_planner.py:569-665``: costmap integral, path length, discounted
goal distance, jerk) of the DEM pose path, and the kinetic energy the
candidate transferred to its ice, which only the DEM gives.

The reference has no DEM rollout; its planners roll the ship out alone
(``jax_mbd_planner.py:51-122``).  Each step of a rollout here is the frame
step of ``jax_simulation.py`` with the controller replaced by the control.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from types import SimpleNamespace
from typing import List, Optional, Sequence

import numpy as np

from . import _abi, sim
from .config import DEFAULT_MATERIAL, IceMaterial

# planner control limits (config.py:390-394) and the action normalisation of
# the MBD planner (jax_mbd_planner.py:2782-2783)
SURGE_MAX, SWAY_MAX, YAW_MAX = 2e6, 5e5, 5e8
ACTION_CENTER = (SURGE_MAX / 2, 0.0, 0.0)
ACTION_SCALE = (SURGE_MAX / 2, SWAY_MAX, YAW_MAX)

_STATIC_ELEM = ("local_polys_padded", "poly_mask", "poly_n_verts", "masses", "inertia", "radii", "areas",
                "thicknesses")
_STATIC_BOND = ("rest_lengths", "bond_strengths", "bond_areas", "sigma_bar_bond")


@dataclass
class RolloutBatch:
    frame_step: object            # multi-system FrameStep (one system per candidate)
    windows: List[np.ndarray]     # field element indices of each candidate's window
    system_start: np.ndarray      # (Q+1,) offsets of the windows in the batch
    sys_start_dev: object         # (Q+1,) int32 device copy
    state: object                 # batched IceState at the rollout start (device)
    ship: object                  # batched ShipState (Q, ...) at the rollout start (device)

    @property
    def n_rollouts(self) -> int:
        return len(self.windows)

    @property
    def n_elements(self) -> int:
        return int(self.system_start[-1])


def sample_controls(rng: np.random.Generator, Q: int, H: int, nominal=(0.0, 0.0), sigma: float = 0.3,
                    surge_max: float = SURGE_MAX, yaw_max: float = YAW_MAX) -> np.ndarray:
    """(H, Q, 3) body-frame controls [X, 0, N]: surge force and yaw moment, each
    Gaussian around its nominal with standard deviation ``sigma`` times its
    maximum, clipped to +-maximum; sway is 0."""
    X = np.clip(rng.normal(nominal[0], sigma * surge_max, (H, Q)), -surge_max, surge_max)
    N = np.clip(rng.normal(nominal[1], sigma * yaw_max, (H, Q)), -yaw_max, yaw_max)
    return np.stack([X, np.zeros_like(X), N], -1)


def predict_paths(eta0, nu0, controls, M3inv, D3, dt: float) -> np.ndarray:
    """Ice-free pose paths (H+1, Q, 3) of the candidates: forward Euler of
    M nu' = tau - D nu and the kinematics, as the DEM's vessel step without ice
    (jax_vessel_dynamics.py:54-84).  Used only to place the windows."""
    H, Q, _ = controls.shape
    eta = np.tile(np.asarray(eta0, np.float64), (Q, 1))
    nu = np.tile(np.asarray(nu0, np.float64), (Q, 1))
    M3inv, D3 = np.asarray(M3inv, np.float64), np.asarray(D3, np.float64)
    out = [eta.copy()]
    for t in range(H):
        nu = nu + dt * ((controls[t] - nu @ D3.T) @ M3inv.T)
        c, s = np.cos(eta[:, 2]), np.sin(eta[:, 2])
        eta = np.stack([eta[:, 0] + dt * (c * nu[:, 0] - s * nu[:, 1]),
                        eta[:, 1] + dt * (s * nu[:, 0] + c * nu[:, 1]), eta[:, 2] + dt * nu[:, 2]], 1)
        out.append(eta.copy())
    return np.stack(out)


def cut_windows(centroids, paths, sizes: Sequence[int], n_samples: int = 5) -> List[np.ndarray]:
    """Window of candidate q: the sizes[q] elements whose centroids lie nearest
    to its path (distance to the nearest of ``n_samples`` points along it),
    sorted by element index."""
    from scipy.spatial import cKDTree
    cents = np.asarray(centroids, np.float64)
    tree = cKDTree(cents)
    H1, Q, _ = paths.shape
    idx_t = np.unique(np.linspace(0, H1 - 1, n_samples).round().astype(int))
    wins = []
    for q in range(Q):
        k = int(min(sizes[q], len(cents)))
        best = {}
        for t in idx_t:
            d, ix = tree.query(paths[t, q, :2], k=k)
            for dd, ii in zip(np.atleast_1d(d), np.atleast_1d(ix)):
                if dd < best.get(ii, np.inf):
                    best[ii] = dd
        items = np.array(list(best.items()), dtype=np.float64)
        order = np.lexsort((items[:, 0], items[:, 1]))[:k]
        wins.append(np.sort(items[order, 0].astype(np.int64)))
    return wins


def window_static(static, windows):
    """Static data of the batch: each window's elements, the bonds with both ends
    inside it and its floes renumbered densely, windows one after another.
    ``static`` holds NumPy arrays (``state.build_static_arrays``)."""
    st = {k: np.asarray(getattr(static, k)) for k in _STATIC_ELEM + _STATIC_BOND + ("bond_i", "bond_j",
                                                                                   "initial_floe_of")}
    n_all = st["masses"].shape[0]
    cols = {k: [] for k in st}
    sys_start, n_off, f_off = [0], 0, 0
    local = -np.ones(n_all, np.int64)
    for w in windows:
        w = np.asarray(w, np.int64)
        local[w] = np.arange(len(w))
        keep = (local[st["bond_i"]] >= 0) & (local[st["bond_j"]] >= 0)
        for k in _STATIC_ELEM:
            cols[k].append(st[k][w])
        for k in _STATIC_BOND:
            cols[k].append(st[k][keep])
        cols["bond_i"].append((local[st["bond_i"][keep]] + n_off).astype(np.int32))
        cols["bond_j"].append((local[st["bond_j"][keep]] + n_off).astype(np.int32))
        _, floe = np.unique(st["initial_floe_of"][w], return_inverse=True)
        cols["initial_floe_of"].append((floe + f_off).astype(np.int32))
        f_off += int(floe.max()) + 1
        n_off += len(w)
        sys_start.append(n_off)
        local[w] = -1
    bs = SimpleNamespace(**{k: np.concatenate(v) for k, v in cols.items()})
    bs.k_n, bs.k_s = float(static.k_n), float(static.k_s)
    bs.pair_i = bs.pair_j = None
    return bs, np.asarray(sys_start, np.int64)


def make_batch(static, ship_dyn, cfg, ship_length: float, ship_beam: float, n_ice_steps: int, dt: float,
               B_mat, T_n: float, positions, windows, eta0, nu0=(0.0, 0.0, 0.0), velocities=None,
               material: IceMaterial = DEFAULT_MATERIAL, dtype=None, device="cuda", **frame_kw) -> RolloutBatch:
    """One system per window, every ship at (eta0, nu0), ice at rest (or at
    ``velocities``), frozen and intact: the state a planner rolls out from."""
    import torch
    from .state import IceState, ShipState
    bs, sys_start = window_static(static, windows)
    fs = sim.make_frame_step(bs, cfg, ship_dyn, ship_length, ship_beam, n_ice_steps, dt, dt / n_ice_steps, False,
                             B_mat, T_n, material=material, device=torch.device(device),
                             dtype=dtype or torch.float32, system_start=sys_start, **frame_kw)
    dev, d = fs.device, fs.dtype
    Q, n, nb, nf = len(windows), fs.n, fs.n_bonds, fs.n_floes
    allw = np.concatenate([np.asarray(w, np.int64) for w in windows])
    pos = torch.as_tensor(np.asarray(positions, np.float64)[allw], dtype=d, device=dev)
    vel = (torch.zeros((n, 2), dtype=d, device=dev) if velocities is None
           else torch.as_tensor(np.asarray(velocities, np.float64)[allw], dtype=d, device=dev))
    z = lambda *s: torch.zeros(s, dtype=d, device=dev)
    state = IceState(positions=pos, velocities=vel, rotations=z(n), angular_vels=z(n), submergence=z(n),
                     bond_intact=torch.ones(nb, dtype=torch.bool, device=dev), bond_damage=z(nb),
                     bond_delta_m_0=z(nb), bond_delta_m_max=z(nb), bond_delta_s=z(nb),
                     elem_active=torch.zeros(n, dtype=torch.bool, device=dev),
                     dpdem_floe_eligible=torch.zeros(nf, dtype=torch.bool, device=dev))
    tile = lambda v, k: torch.as_tensor(np.tile(np.asarray(v, np.float64), (Q, 1)), dtype=d, device=dev)
    ship = ShipState(eta=tile(eta0, 3), nu=tile(nu0, 3), n_actual=z(Q, 6), e_int=z(Q, 3))
    if Q == 1:  # a single system takes unbatched ship arrays
        ship = ShipState(*[t[0] for t in ship])
    ss = torch.as_tensor(sys_start, dtype=torch.int32, device=dev)
    return RolloutBatch(fs, [np.asarray(w) for w in windows], sys_start, ss, state, ship)


@dataclass
class RolloutResult:
    state: object      # IceState after H steps
    ship: object       # ShipState (Q, ...) after H steps
    history: tuple     # the segment history (poses (H, Q, 3) at index 3)
    controls: object   # (H, Q, 3) device controls


def run(batch: RolloutBatch, controls, v_water=None, history=True, check: bool = True) -> RolloutResult:
    """All H steps of all candidates in one launch (``dem_rollout_segment``).
    ``controls`` (H, Q, 3); ``v_water`` (H, n, 2) or None (still water);
    ``history="ship"`` records the ship rows only (what ``costs`` reads)."""
    import torch
    fs = batch.frame_step
    u = sim._as_tensor(controls, fs.dtype, fs.device)
    H = int(u.shape[0])
    if fs.n_systems == 1 and u.dim() == 3:  # (H, 1, 3) -> (H, 3) for a single system
        u = u.reshape(H, 3)
    vw = (torch.zeros((H, fs.n, 2), dtype=fs.dtype, device=fs.device) if v_water is None
          else sim._as_tensor(v_water, fs.dtype, fs.device))
    fin, ship, hist = fs.rollout_segment(batch.state, batch.ship, u, vw, None, history=history, check=check)
    return RolloutResult(fin, ship, hist, u)


def costs(batch: RolloutBatch, result: RolloutResult, costmap, goal_xy, ship_length: float = 0.0,
          ship_beam: float = 0.0, action_center=ACTION_CENTER, action_scale=ACTION_SCALE,
          oob_penalty: float = 1e8, cost_truncate_y: Optional[float] = None, out=None):
    """(Q, 5) float64 device tensor per candidate: [costmap integral, path length,
    goal distance, jerk, transferred ice kinetic energy] (``dem_rollout_costs``).

    ``costmap`` is a ``JaxCostMapResult`` with its device grid (``costmap.
    build_costmap_jax``); ``ship_length``/``ship_beam`` > 0 query the hull
    centre and corners as the planner does with its hull dimensions."""
    fs = batch.frame_step
    Q, H = batch.n_rollouts, int(result.controls.shape[0])
    return path_costs(batch.ship.eta.reshape(Q, 3), result.history[3].reshape(H, Q, 3),
                      result.controls.reshape(H, Q, 3), costmap, goal_xy, ship_length, ship_beam,
                      action_center, action_scale, oob_penalty, cost_truncate_y, masses=fs._keep["masses"],
                      vel0=batch.state.velocities, vel1=result.state.velocities, system_start=batch.sys_start_dev,
                      out=out)


def _device_grid(costmap):
    import torch
    grid = costmap.grid
    if grid is None or not grid.is_cuda or grid.dtype != torch.float32:
        raise ValueError("costmap.grid must be the float32 device grid")
    return grid.contiguous()


def _cost_params(costmap, oob_penalty, ship_length, ship_beam, goal_xy=(0.0, 0.0), action_center=ACTION_CENTER,
                 action_scale=ACTION_SCALE, cost_truncate_y=None):
    return _abi.DemRolloutCostParams(
        x_origin=costmap.x_origin, y_origin=costmap.y_origin, resolution=costmap.resolution, rows=costmap.rows,
        cols=costmap.cols, oob_penalty=oob_penalty, ship_length=ship_length, ship_beam=ship_beam,
        goal_x=float(goal_xy[0]), goal_y=float(goal_xy[1]),
        action_center=(C.c_double * 3)(*[float(v) for v in action_center]),
        action_scale=(C.c_double * 3)(*[float(v) for v in action_scale]),
        has_truncate=0 if cost_truncate_y is None else 1, reserved=0,
        truncate_y=0.0 if cost_truncate_y is None else float(cost_truncate_y))


def waypoint_costs(eta_hist, costmap, ship_length: float = 0.0, ship_beam: float = 0.0, oob_penalty: float = 1e8,
                   out=None):
    """``dem_rollout_waypoint_costs``: (Q, H) float32 costmap value of each
    pose of the paths eta_hist (H, Q, 3) (hull centre and box corners, max)."""
    import torch
    lib = _abi.load_library()
    eta_hist = eta_hist.contiguous()
    dt = eta_hist.dtype
    if dt not in (torch.float32, torch.float64) or eta_hist.dim() != 3 or eta_hist.shape[2] != 3:
        raise ValueError("eta_hist must be (H,Q,3) float32 or float64")
    H, Q = int(eta_hist.shape[0]), int(eta_hist.shape[1])
    grid = _device_grid(costmap)
    P = _cost_params(costmap, oob_penalty, ship_length, ship_beam)
    if out is None:
        out = torch.empty((Q, H), dtype=torch.float32, device=eta_hist.device)
    rc = lib.dem_rollout_waypoint_costs(_abi.DEM_F64 if dt == torch.float64 else _abi.DEM_F32, Q, H,
                                        eta_hist.data_ptr(), grid.data_ptr(), C.byref(P), out.data_ptr(),
                                        C.c_void_p(torch.cuda.current_stream(eta_hist.device).cuda_stream))
    if rc != _abi.DEM_OK:
        raise _abi.DemError(rc, "dem_rollout_waypoint_costs failed")
    return out


def path_costs(eta0, eta_hist, controls, costmap, goal_xy, ship_length: float = 0.0, ship_beam: float = 0.0,
               action_center=ACTION_CENTER, action_scale=ACTION_SCALE, oob_penalty: float = 1e8,
               cost_truncate_y: Optional[float] = None, masses=None, vel0=None, vel1=None, system_start=None,
               out=None):
    """``dem_rollout_costs`` on device tensors: pose paths eta0 (Q,3) + eta_hist
    (H,Q,3), physical controls (H,Q,3) or None, a costmap with ``grid``,
    ``x_origin``, ``y_origin``, ``resolution``, ``rows``, ``cols``; with masses,
    vel0, vel1 and system_start also the transferred kinetic energy."""
    import torch
    lib = _abi.load_library()
    eta0 = eta0.contiguous()
    eta_hist = eta_hist.contiguous()
    dev, dt = eta0.device, eta0.dtype
    if dt not in (torch.float32, torch.float64) or eta_hist.dtype != dt:
        raise ValueError("poses must share one float dtype")
    Q = int(eta0.shape[0])
    H = int(eta_hist.shape[0])
    if tuple(eta0.shape) != (Q, 3) or tuple(eta_hist.shape) != (H, Q, 3):
        raise ValueError("eta0 must be (Q,3) and eta_hist (H,Q,3)")
    if controls is not None:
        controls = controls.to(dev, dt).contiguous()
        if tuple(controls.shape) != (H, Q, 3):
            raise ValueError("controls must be (H,Q,3)")
    grid = _device_grid(costmap)
    P = _cost_params(costmap, oob_penalty, ship_length, ship_beam, goal_xy, action_center, action_scale,
                     cost_truncate_y)
    ke = masses is not None
    if ke:
        masses, vel0, vel1 = (t.to(dev, dt).contiguous() for t in (masses, vel0, vel1))
        system_start = system_start.to(dev, torch.int32).contiguous()
    if out is None:
        out = torch.empty((Q, 5), dtype=torch.float64, device=dev)
    p = lambda t: None if t is None else t.data_ptr()
    rc = lib.dem_rollout_costs(_abi.DEM_F64 if dt == torch.float64 else _abi.DEM_F32, Q, H, p(system_start),
                               p(eta0), p(eta_hist), p(controls), p(grid), C.byref(P), p(masses), p(vel0), p(vel1),
                               p(out), C.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    if rc != _abi.DEM_OK:
        raise _abi.DemError(rc, "dem_rollout_costs failed")
    return out


# ─── the planner-rollout workload ────────────────────────────────────────────

@dataclass
class PlannerWorkload:
    batch: RolloutBatch
    controls: np.ndarray   # (H, Q, 3)
    costmap: object        # JaxCostMapResult (256 x 256, 2 m cells)
    goal: np.ndarray       # (2,)
    ship_length: float
    ship_beam: float


def planner_workload(field, Q: int = 2048, H: int = 64, seed: int = 0, min_elements: int = 200,
                     max_elements: int = 3000, eta0=None, speed: float = 2.0, costmap_cells: int = 256,
                     dtype=None, device="cuda", **frame_kw) -> PlannerWorkload:
    """Q candidate rollouts of H control steps from one ship state in ``field``.

    Controls: surge force and yaw moment Gaussian around their nominal (the
    surge force holding ``speed`` against linear damping, zero yaw moment) with
    sigma 0.3 of their maxima.  Windows: log-uniform sizes in
    [min_elements, max_elements], the elements nearest each candidate's
    ice-free predicted path.  Costmap: the KE costmap of the field,
    ``costmap_cells`` square 2 m cells centred on the start.  Goal: 200 m ahead."""
    import torch
    from .config import get_default_simulation_config
    from .costmap import build_costmap_jax
    from .state import build_static_arrays, ship_dynamics_arrays
    from .vessel import SupplyVessel
    rng = np.random.default_rng(seed)
    cfg = get_default_simulation_config()
    static = build_static_arrays(field.polygons, field.centroids, field.bonds, field.thicknesses,
                                 field.parent_ids, cfg, DEFAULT_MATERIAL, 0.05)
    sd = ship_dynamics_arrays(field.ship_props, cfg, field.ship_length, field.ship_beam, field.hull_local)
    if eta0 is None:
        eta0 = ice_edge_pose(field)
    eta0 = np.asarray(eta0, np.float64)
    nu0 = np.array([speed, 0.0, 0.0])
    x_nom = float(np.clip((np.asarray(sd.D3) @ nu0)[0], -SURGE_MAX, SURGE_MAX))
    u = sample_controls(rng, Q, H, nominal=(x_nom, 0.0))
    paths = predict_paths(eta0, nu0, u, sd.M3inv, sd.D3, field.dt)
    sizes = np.exp(rng.uniform(np.log(min_elements), np.log(max_elements), Q)).astype(np.int64)
    wins = cut_windows(field.centroids, paths, sizes)
    sv = SupplyVessel(mass=field.ship_props.mass, length=field.ship_length)
    sd_dev = sim_ship_dyn(sd, dtype or torch.float32, device)
    batch = make_batch(static, sd_dev, cfg, field.ship_length, field.ship_beam, field.n_ice_steps, field.dt, sv.B,
                       sv.T_n, field.centroids, wins, eta0, nu0, dtype=dtype, device=device, **frame_kw)
    half = 0.5 * costmap_cells * 2.0 - 20.0  # 2 m cells with the builder's 20 m margin
    cm, _ = build_costmap_jax(field.centroids, field.thicknesses, static.radii, eta0[0] - half, eta0[0] + half,
                              eta0[1] - half, eta0[1] + half, resolution=2.0, ship_length=field.ship_length,
                              ship_beam=field.ship_beam, masses=static.masses, device=device, download=False)
    goal = eta0[:2] + 200.0 * np.array([np.cos(eta0[2]), np.sin(eta0[2])])
    return PlannerWorkload(batch, u, cm, goal, field.ship_length, field.ship_beam)


def ice_edge_pose(field, gap: float = 3.0) -> np.ndarray:
    """Pose on the field's ship track, heading as the track, with the bow ``gap``
    metres short of the nearest element centroid ahead within half a beam."""
    p = np.asarray(field.trajectory[0], np.float64)
    d = np.array([np.cos(p[2]), np.sin(p[2])])
    rel = np.asarray(field.centroids, np.float64) - p[:2]
    along = rel @ d
    across = np.abs(rel @ np.array([-d[1], d[0]]))
    ahead = along[(along > 0) & (across < 0.5 * field.ship_beam)]
    if len(ahead) == 0:
        return p
    s = float(ahead.min()) - 0.5 * field.ship_length - gap
    return np.array([p[0] + s * d[0], p[1] + s * d[1], p[2]])


def sim_ship_dyn(sd, dtype, device):
    """Ship dynamics arrays on the device (``ShipDynamicsData`` of tensors)."""
    from .state import to_device
    return to_device(sd, dtype, device)
