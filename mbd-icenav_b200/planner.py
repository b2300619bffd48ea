"""Model-based-diffusion planning with the DEM in the loop, plain and
surrogate-screened.

``mbd_plan`` mirrors the reference's ``run_mbd`` (``jax_mbd_planner.py:
1314-1411``): a mean action sequence Ybar (H, 2) in normalised action space
(surge force, yaw moment) is refined over ``n_diffuse - 1`` reverse diffusion
steps; each step draws ``n_sample`` candidates Y0 = clip(Ybar + sigma_i eps),
scores them with a cost batch, and moves Ybar to the softmax(-cost / T)
weighted mean through the same score update.  Sway is held at zero (the
surrogate's controls are (surge, yaw) per step).

Two cost batches:

* ``DemScorer`` — every candidate rolled out by the DEM (``dem_rollout_segment``,
  one system per candidate, each its own copy of the ice window around the
  start) and scored on the device: the reference planner's cost components
  (``dem_rollout_costs``) plus the ice terms only the DEM gives (kinetic energy
  transferred, hull impulse, bonds broken; ``dem_rollout_ice_terms``);
* ``ScreenedScorer`` — the rigid-ship rollout (``dem_ship_rollout``) for the
  planner's components plus the surrogate's prediction of the ice terms for
  every candidate; the ``top_k`` best and a random check set are re-scored by
  the DEM and only they keep a cost.  When the check set beats the screened
  best by more than ``max_rel_err``, the step falls back to scoring every
  candidate with the DEM.

The reference has no DEM rollout and no surrogate; its planners score
rigid-ship rollouts on a static costmap.  Torch tensors hold the device
buffers; the planner's bookkeeping (sampling, softmax, weighted mean) uses
torch tensor ops as the reference uses jnp.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field as dc_field
from types import SimpleNamespace
from typing import List, Optional

import numpy as np

from . import _abi, rollouts, sg_ops, sim
from . import surrogate as S
from .config import DEFAULT_MATERIAL

_torch = None


def _tm():
    global _torch
    if _torch is None:
        import torch
        _torch = torch
    return _torch


# ─── cost ───────────────────────────────────────────────────────────────────
@dataclass
class CostWeights:
    """J = costmap / normalizer * w_costmap + w_length * length + w_goal * goal
    + w_jerk * jerk (the reference's weighted components, jax_mbd_planner.py:
    668-717, with its planner defaults) + the DEM's ice terms."""
    w_costmap: float = 1.0
    costmap_normalizer: float = 1.0
    w_length: float = 0.0
    w_goal: float = 0.0
    w_jerk: float = 0.0
    w_ke: float = 1e-3       # per J of kinetic energy transferred to the ice
    w_impulse: float = 1e-4  # per N s of hull impulse
    w_bonds: float = 1.0     # per bond broken

    def planner(self):
        return (self.w_costmap / self.costmap_normalizer, self.w_length, self.w_goal, self.w_jerk)

    def ice(self):
        return (self.w_ke, self.w_impulse, self.w_bonds)


@dataclass
class MBDConfig:
    horizon: int = 64
    n_sample: int = 8192
    n_diffuse: int = 17          # 16 reverse steps
    temperature: float = 0.01    # config.py planning_jax_mbd_temperature
    beta0: float = 1e-5
    betaT: float = 0.05
    init_surge_bias: float = 0.7
    top_k: int = 64
    max_rel_err: float = 0.05


# ─── the scene a plan starts from ───────────────────────────────────────────
@dataclass
class PlanScene:
    field: object
    static: object           # NumPy static arrays of the whole field
    ship_dyn: object         # NumPy ship dynamics arrays
    eta0: np.ndarray
    nu0: np.ndarray
    window: np.ndarray       # field element indices within reach of every candidate
    costmap: object          # JaxCostMapResult, device grid, centred on the start
    patch: object            # (1, 64, 64, 1) bf16 normalised costmap patch around the start
    goal: np.ndarray
    params: object           # DemParams (vessel constants for the rigid rollout)
    dtype: object
    device: object
    sweep: object = None     # device inputs of dem_rollout_sweep_features (``sweep_inputs``)


PATCH_CELLS = S.PATCH
COSTMAP_CELLS = 256
RESOLUTION = 2.0


def reach_radius(field, horizon: int, dt: float, v_max: float = 5.0) -> float:
    """Distance from the start within which any candidate's hull can touch ice."""
    return math.hypot(0.5 * field.ship_length, 0.5 * field.ship_beam) + v_max * horizon * dt + 5.0


def make_scene(field, eta0, nu0=(2.0, 0.0, 0.0), horizon: int = 64, dtype=None, device="cuda",
               patch_stats=(0.0, 1.0), static=None, ship_dyn=None, removed=None) -> PlanScene:
    """The plan's start: the window of elements any candidate can reach, the
    costmap around the start and its normalised patch.  ``removed``: element
    indices that are not in the scene (the channel a transiting ship has
    cleared behind and around it); they are left out of the window and the
    costmap."""
    torch = _tm()
    from .config import get_default_simulation_config
    from .costmap import build_costmap_jax
    from .state import build_static_arrays, ship_dynamics_arrays
    from .vessel import SupplyVessel
    cfg = get_default_simulation_config()
    dev = torch.device(device)
    dtype = dtype or torch.float32
    if static is None:
        static = build_static_arrays(field.polygons, field.centroids, field.bonds, field.thicknesses,
                                     field.parent_ids, cfg, DEFAULT_MATERIAL, 0.05)
    if ship_dyn is None:
        ship_dyn = ship_dynamics_arrays(field.ship_props, cfg, field.ship_length, field.ship_beam, field.hull_local)
    eta0 = np.asarray(eta0, np.float64)
    nu0 = np.asarray(nu0, np.float64)
    R = reach_radius(field, horizon, field.dt)
    d = np.linalg.norm(np.asarray(field.centroids, np.float64) - eta0[:2], axis=1)
    present = np.ones(len(d), bool)
    if removed is not None:
        present[np.asarray(removed, np.int64)] = False
    window = np.nonzero((d < R) & present)[0]
    half = 0.5 * COSTMAP_CELLS * RESOLUTION - 20.0  # 256 cells with the builder's 20 m margin
    cents = np.asarray(field.centroids, np.float64)
    near = present & (np.abs(cents[:, 0] - eta0[0]) < half + 60.0) & (np.abs(cents[:, 1] - eta0[1]) < half + 60.0)
    thick = np.asarray(field.thicknesses, np.float64)
    cm, _ = build_costmap_jax(cents[near], thick[near], np.asarray(static.radii)[near], eta0[0] - half,
                              eta0[0] + half, eta0[1] - half, eta0[1] + half, resolution=RESOLUTION,
                              ship_length=field.ship_length, ship_beam=field.ship_beam,
                              masses=np.asarray(static.masses)[near], device=dev, download=False)
    c0 = (COSTMAP_CELLS - PATCH_CELLS) // 2
    mean, std = patch_stats
    patch32 = ((cm.grid[c0:c0 + PATCH_CELLS, c0:c0 + PATCH_CELLS] - mean) / std).contiguous()
    patch = sg_ops.to_bf16(patch32).view(1, PATCH_CELLS, PATCH_CELLS, 1)
    sv = SupplyVessel(mass=field.ship_props.mass, length=field.ship_length)
    P = sim.build_params(cfg, ship_dyn, field.ship_length, field.ship_beam, field.n_ice_steps, field.dt,
                         field.dt / field.n_ice_steps, False, sv.B, sv.T_n)
    goal = eta0[:2] + 200.0 * np.array([math.cos(eta0[2]), math.sin(eta0[2])])
    return PlanScene(field, static, ship_dyn, eta0, nu0, window, cm, patch, goal, P, dtype, dev)


def shared_window_batch(scene: PlanScene, Q: int, **frame_kw) -> rollouts.RolloutBatch:
    """Q systems, each its own copy of the scene's window (the candidates of one plan)."""
    torch = _tm()
    from .state import IceState, ShipState
    from .vessel import SupplyVessel
    from .config import get_default_simulation_config
    f = scene.field
    st = scene.static
    w = np.asarray(scene.window, np.int64)
    n_w = len(w)
    local = -np.ones(st.masses.shape[0], np.int64)
    local[w] = np.arange(n_w)
    bi, bj = np.asarray(st.bond_i, np.int64), np.asarray(st.bond_j, np.int64)
    keep = (local[bi] >= 0) & (local[bj] >= 0)
    nb_w = int(keep.sum())
    _, floe = np.unique(np.asarray(st.initial_floe_of)[w], return_inverse=True)
    nf_w = int(floe.max()) + 1 if n_w else 0
    tile = lambda a: np.concatenate([np.asarray(a)] * Q, axis=0)
    bs = SimpleNamespace()
    for k in rollouts._STATIC_ELEM:
        setattr(bs, k, tile(np.asarray(getattr(st, k))[w]))
    for k in rollouts._STATIC_BOND:
        setattr(bs, k, tile(np.asarray(getattr(st, k))[keep]))
    offs_e = (np.arange(Q, dtype=np.int64) * n_w)[:, None]
    bs.bond_i = (local[bi[keep]][None, :] + offs_e).reshape(-1).astype(np.int32)
    bs.bond_j = (local[bj[keep]][None, :] + offs_e).reshape(-1).astype(np.int32)
    bs.initial_floe_of = (floe[None, :] + (np.arange(Q) * nf_w)[:, None]).reshape(-1).astype(np.int32)
    bs.k_n, bs.k_s = float(st.k_n), float(st.k_s)
    bs.pair_i = bs.pair_j = None
    sys_start = np.arange(Q + 1, dtype=np.int64) * n_w
    cfg = get_default_simulation_config()
    sv = SupplyVessel(mass=f.ship_props.mass, length=f.ship_length)
    sd_dev = rollouts.sim_ship_dyn(scene.ship_dyn, scene.dtype, scene.device)
    fs = sim.make_frame_step(bs, cfg, sd_dev, f.ship_length, f.ship_beam, f.n_ice_steps, f.dt,
                             f.dt / f.n_ice_steps, False, sv.B, sv.T_n, device=scene.device, dtype=scene.dtype,
                             system_start=sys_start if Q > 1 else None, **frame_kw)
    dev, d = fs.device, fs.dtype
    n, nb, nf = fs.n, fs.n_bonds, fs.n_floes
    pos = torch.as_tensor(np.asarray(f.centroids, np.float64)[w], dtype=d, device=dev).repeat(Q, 1)
    z = lambda *s: torch.zeros(s, dtype=d, device=dev)
    state = IceState(positions=pos, velocities=z(n, 2), rotations=z(n), angular_vels=z(n), submergence=z(n),
                     bond_intact=torch.ones(nb, dtype=torch.bool, device=dev), bond_damage=z(nb),
                     bond_delta_m_0=z(nb), bond_delta_m_max=z(nb), bond_delta_s=z(nb),
                     elem_active=torch.zeros(n, dtype=torch.bool, device=dev),
                     dpdem_floe_eligible=torch.zeros(nf, dtype=torch.bool, device=dev))
    tq = lambda v: torch.as_tensor(np.tile(np.asarray(v, np.float64), (Q, 1)), dtype=d, device=dev)
    ship = ShipState(eta=tq(scene.eta0), nu=tq(scene.nu0), n_actual=z(Q, 6), e_int=z(Q, 3))
    if Q == 1:
        ship = ShipState(*[t[0] for t in ship])
    batch = rollouts.RolloutBatch(fs, [w] * Q, sys_start, torch.as_tensor(sys_start, dtype=torch.int32, device=dev),
                                  state, ship)
    batch.bond_start = torch.as_tensor(np.arange(Q + 1) * nb_w, dtype=torch.int32, device=dev)
    return batch


# ─── controls and features ──────────────────────────────────────────────────
def physical_controls(Yn):
    """(Q, H, 2) normalised (surge, yaw) in [-1, 1] -> (H, Q, 3) body-frame [X, 0, N]."""
    torch = _tm()
    c, s = rollouts.ACTION_CENTER, rollouts.ACTION_SCALE
    X = c[0] + s[0] * Yn[..., 0]
    N = c[2] + s[2] * Yn[..., 1]
    return torch.stack([X, torch.zeros_like(X), N], -1).transpose(0, 1).contiguous()


# scales of the sweep features before log1p: elements, kg, J, N s, kg, J, bonds, bonds
SWEEP_SCALE = (1.0, 1e3, 1e3, 1e3, 1e3, 1e3, 1.0, 1.0)


def features(scene: PlanScene, Yn, wcost, sweep):
    """(Q, 6 + 3H + 8) fp32 network inputs besides the patch: ship state [u/5,
    v/2, r/0.1, cos psi, sin psi, 0], the normalised controls step by step,
    log1p of ``wcost`` (Q, H), the costmap value at each pose of the
    candidate's rigid-ship path, and log1p of ``sweep`` (Q, 8), what that path
    sweeps through the ice window, over ``SWEEP_SCALE`` (both from
    ``rigid_path``)."""
    torch = _tm()
    Q, H, _ = Yn.shape
    e, v = scene.eta0, scene.nu0
    ship = torch.tensor([v[0] / 5.0, v[1] / 2.0, v[2] / 0.1, math.cos(e[2]), math.sin(e[2]), 0.0],
                        dtype=torch.float32, device=Yn.device)
    path = torch.log1p(torch.clamp(wcost.float(), min=0.0))
    sc = torch.tensor(SWEEP_SCALE, dtype=torch.float32, device=Yn.device)
    sw = torch.log1p(torch.clamp(sweep.float(), min=0.0) / sc)
    return torch.cat([ship.expand(Q, S.N_SHIP), Yn.reshape(Q, 2 * H).float(), path, sw], 1).contiguous()


# ─── target transforms ──────────────────────────────────────────────────────
TARGET_SCALE = (1e3, 1e3, 1.0)  # J, N s, bonds: log1p(x / scale) before standardising


@dataclass
class TargetStats:
    mean: np.ndarray
    std: np.ndarray

    def forward(self, raw):
        """raw (Q, 3) -> standardised log1p targets (torch, fp32)."""
        torch = _tm()
        sc = torch.tensor(TARGET_SCALE, dtype=torch.float64, device=raw.device)
        t = torch.log1p(torch.clamp(raw.double(), min=0.0) / sc)
        m = torch.as_tensor(self.mean, device=raw.device)
        s = torch.as_tensor(self.std, device=raw.device)
        return ((t - m) / s).float()

    def inverse(self, pred):
        torch = _tm()
        sc = torch.tensor(TARGET_SCALE, dtype=torch.float64, device=pred.device)
        m = torch.as_tensor(self.mean, device=pred.device)
        s = torch.as_tensor(self.std, device=pred.device)
        return torch.clamp(torch.expm1(pred.double() * s + m), min=0.0) * sc


# ─── scorers ────────────────────────────────────────────────────────────────
class DemScorer:
    """Every candidate through the batched DEM."""

    def __init__(self, scene: PlanScene, Q: int, weights: CostWeights, **frame_kw):
        self.scene = scene
        self.Q = Q
        self.w = weights
        self.batch = shared_window_batch(scene, Q, **frame_kw)
        torch = _tm()
        self.cost_out = torch.empty((Q, 5), dtype=torch.float64, device=scene.device)
        self.ice_out = torch.empty((Q, 2), dtype=torch.float64, device=scene.device)
        self.rollouts = 0

    def terms(self, Yn):
        """(Q, 7) float64: [costmap, length, goal, jerk, KE, impulse, bonds] of the candidates."""
        torch = _tm()
        sc = self.scene
        u = physical_controls(Yn).to(sc.dtype)
        res = rollouts.run(self.batch, u, history="ship", check=True)
        comp = rollouts.costs(self.batch, res, sc.costmap, sc.goal, sc.field.ship_length, sc.field.ship_beam,
                              out=self.cost_out)
        fs = self.batch.frame_step
        H = int(u.shape[0])
        rc = fs.lib.dem_rollout_ice_terms(_abi.DEM_F64 if fs.dtype == torch.float64 else _abi.DEM_F32, self.Q, H,
                                          res.history[5].data_ptr(), self.batch.bond_start.data_ptr(),
                                          self.batch.state.bond_intact.data_ptr(),
                                          res.state.bond_intact.data_ptr(), self.ice_out.data_ptr(),
                                          fs._stream())
        if rc != _abi.DEM_OK:
            raise _abi.DemError(rc, "dem_rollout_ice_terms failed")
        self.rollouts += self.Q
        return torch.cat([comp[:, :4], comp[:, 4:5], self.ice_out], 1)

    def autotune(self, Yn):
        """Pick this batch's work split by timing it on candidates Yn (every
        choice gives identical results); returns (choice, {choice: ms})."""
        from . import autotune
        u = physical_controls(Yn).to(self.scene.dtype)
        return autotune.tune(self.batch.frame_step, lambda: rollouts.run(self.batch, u, history="ship", check=False))

    def total(self, terms):
        torch = _tm()
        w = torch.tensor(self.w.planner() + self.w.ice(), dtype=torch.float64, device=terms.device)
        return terms @ w

    def __call__(self, Yn):
        return self.total(self.terms(Yn))


class Surrogate:
    """A trained ``SurrogateNet`` with its input and target normalisation."""

    def __init__(self, net: S.SurrogateNet, stats: TargetStats, patch_stats=(0.0, 1.0)):
        self.net = net
        self.stats = stats
        self.patch_stats = patch_stats

    def predict(self, scene: PlanScene, Yn):
        """(Q, 3) float64 predicted ice terms [KE, impulse, bonds] of the
        candidates (their rigid-ship paths from ``rigid_path``)."""
        _, wcost, sweep = rigid_path(scene, Yn)
        return self.predict_features(scene, features(scene, Yn, wcost, sweep))

    def predict_features(self, scene: PlanScene, ext):
        """``predict`` from the candidates' ``features`` rows (Q, 6 + 3H)."""
        torch = _tm()
        Q = int(ext.shape[0])
        enc = self.net.encode(scene.patch, tag="plan_enc")
        rows = self.net._buf("plan_rows", (Q,), torch.int32)
        rows.zero_()
        out = self.net.head(enc, ext, enc_row=rows, tag="plan_head")
        return self.stats.inverse(out[:, :S.N_OUT])


def rigid_terms(scene: PlanScene, Yn, out=None):
    """(Q, 4) float64 planner components of the rigid-ship paths (``dem_ship_rollout``)."""
    return rigid_path(scene, Yn, out)[0]


def sweep_inputs(scene: PlanScene):
    """The window's elements (start positions, radii, masses) and its bonds in
    window indices, on the device (cached on the scene)."""
    if scene.sweep is not None:
        return scene.sweep
    torch = _tm()
    st = scene.static
    w = np.asarray(scene.window, np.int64)
    local = -np.ones(np.asarray(st.masses).shape[0], np.int64)
    local[w] = np.arange(len(w))
    bi, bj = np.asarray(st.bond_i, np.int64), np.asarray(st.bond_j, np.int64)
    keep = (local[bi] >= 0) & (local[bj] >= 0)
    dev, d = scene.device, scene.dtype
    scene.sweep = SimpleNamespace(
        n=len(w), nb=int(keep.sum()),
        pos=torch.as_tensor(np.asarray(scene.field.centroids, np.float64)[w], dtype=d, device=dev).contiguous(),
        radii=torch.as_tensor(np.asarray(st.radii, np.float64)[w], dtype=d, device=dev),
        masses=torch.as_tensor(np.asarray(st.masses, np.float64)[w], dtype=d, device=dev),
        bi=torch.as_tensor(local[bi[keep]], dtype=torch.int32, device=dev),
        bj=torch.as_tensor(local[bj[keep]], dtype=torch.int32, device=dev))
    return scene.sweep


def sweep_features(scene: PlanScene, eta0, hist):
    """``dem_rollout_sweep_features``: (Q, 8) float32, what each pose path
    eta0 (Q, 3), hist (H, Q, 3) sweeps through the scene's ice window."""
    torch = _tm()
    lib = _abi.load_library()
    H, Q, _ = hist.shape
    w = sweep_inputs(scene)
    out = torch.empty((Q, S.N_SWEEP), dtype=torch.float32, device=hist.device)
    f = scene.field
    rc = lib.dem_rollout_sweep_features(_abi.DEM_F64 if hist.dtype == torch.float64 else _abi.DEM_F32, Q, H,
                                        eta0.data_ptr(), hist.data_ptr(), w.n, w.pos.data_ptr(),
                                        w.radii.data_ptr(), w.masses.data_ptr(), w.nb, w.bi.data_ptr(),
                                        w.bj.data_ptr(), 0.5 * f.ship_length, 0.5 * f.ship_beam, float(f.dt),
                                        out.data_ptr(), torch.cuda.current_stream(hist.device).cuda_stream)
    if rc != _abi.DEM_OK:
        raise _abi.DemError(rc, "dem_rollout_sweep_features failed")
    return out


def rigid_path(scene: PlanScene, Yn, out=None):
    """The candidates' rigid-ship paths (``dem_ship_rollout``): their (Q, 4)
    float64 planner components, the (Q, H) float32 costmap value at each pose
    (``dem_rollout_waypoint_costs``) and the (Q, 8) float32 sweep features
    (``sweep_features``)."""
    torch = _tm()
    lib = _abi.load_library()
    Q, H, _ = Yn.shape
    d = scene.dtype
    u = physical_controls(Yn).to(d)
    eta0 = torch.as_tensor(np.tile(scene.eta0, (Q, 1)), dtype=d, device=scene.device)
    nu0 = torch.as_tensor(np.tile(scene.nu0, (Q, 1)), dtype=d, device=scene.device)
    hist = torch.empty((H, Q, 3), dtype=d, device=scene.device)
    import ctypes as C
    rc = lib.dem_ship_rollout(C.byref(scene.params), _abi.DEM_F64 if d == torch.float64 else _abi.DEM_F32, Q, H,
                              eta0.data_ptr(), nu0.data_ptr(), u.data_ptr(), None, hist.data_ptr(), None,
                              C.c_void_p(torch.cuda.current_stream(scene.device).cuda_stream))
    if rc != _abi.DEM_OK:
        raise _abi.DemError(rc, "dem_ship_rollout failed")
    comp = rollouts.path_costs(eta0, hist, u, scene.costmap, scene.goal, scene.field.ship_length,
                               scene.field.ship_beam, out=out)
    wcost = rollouts.waypoint_costs(hist, scene.costmap, scene.field.ship_length, scene.field.ship_beam)
    return comp[:, :4], wcost, sweep_features(scene, eta0, hist)


class ScreenedScorer:
    """Surrogate predictions for every candidate, the DEM for the best ``top_k``
    and for ``n_check`` random others.

    The ``top_k`` candidates the surrogate ranks best are rolled out by the DEM
    together with ``n_check`` candidates drawn at random from the rest (the
    held-out check).  Only these keep a cost, their exact DEM cost; every other
    candidate gets +inf (weight 0 in the MBD softmax), so no cost the DEM has
    not checked can win a step.  The check of a step is the relative amount by
    which the best random candidate beats the best screened one (0 when it
    does not): screening that misses better candidates than it keeps shows up
    there.  Above ``max_rel_err`` the step falls back to scoring every
    candidate with the plain DEM.

    With ``deepen`` > 0 the check is split: half of it is drawn from the band
    of the ``deepen`` candidates ranked just below the top_k, half from the
    rest.  When the band sample beats the screened best by more than
    ``max_rel_err`` (but the rest does not), the DEM scores the whole band too
    and those candidates keep their exact costs (``deepened`` counts such
    steps): a ranking that misses near its cut costs a band instead of the
    whole population.  A miss in the rest still falls back.

    With ``adapt_steps`` > 0 the network also learns the scene as the plan
    goes: after each step, that many Adam steps (batches of up to 256,
    learning rate ``adapt_lr``) on the step's unbiased DEM samples, whose exact
    ice terms the step has anyway: the random check set, or every candidate
    after a fallback.  (The screened top-k are the network's own picks;
    training on them teaches it that its picks are good.)  ``restore`` puts
    back the network the scorer started from."""

    def __init__(self, scene: PlanScene, surrogate: Surrogate, Q: int, weights: CostWeights, top_k: int = 64,
                 max_rel_err: float = 0.05, n_check: int = 64, seed: int = 0, adapt_steps: int = 0,
                 adapt_lr: float = 3e-4, deepen: int = 0, **frame_kw):
        torch = _tm()
        self.scene = scene
        self.sur = surrogate
        self.w = weights
        self.Q = Q
        self.k = top_k
        self.n_check = max(0, min(n_check, Q - top_k))
        self.deepen = max(0, min(int(deepen), Q - top_k - (self.n_check + 1) // 2))
        self.n_band = min(self.n_check // 2, self.deepen)  # band part of the check
        self.dem_band = None
        self.deepened = 0
        self.band_errs: List[float] = []   # per step: how much the best band sample beats the screened best
        self.max_rel_err = max_rel_err
        self.dem_k = DemScorer(scene, top_k + self.n_check, weights, **frame_kw)
        self.dem_all = None
        self.frame_kw = frame_kw
        self.gen = torch.Generator(device=scene.device).manual_seed(seed)
        self.fallbacks = 0
        self.rel_errs: List[float] = []    # per step: how much the best random candidate beats the screened best
        self.pred_errs: List[float] = []   # per step: mean relative error of the predicted totals (top_k)
        self.rollouts = 0
        self.adapt_steps = int(adapt_steps)
        self.adapt_lr = float(adapt_lr)
        self._base = surrogate.net.state() if self.adapt_steps > 0 else None
        self._ext = None
        self._pat = None

    def predicted(self, Yn):
        """(Q,) float64 predicted totals: rigid-path planner terms + predicted ice terms."""
        torch = _tm()
        planner, wcost, sweep = rigid_path(self.scene, Yn)
        self._ext = features(self.scene, Yn, wcost, sweep)
        ice = self.sur.predict_features(self.scene, self._ext)
        wp = torch.tensor(self.w.planner(), dtype=torch.float64, device=Yn.device)
        wi = torch.tensor(self.w.ice(), dtype=torch.float64, device=Yn.device)
        return planner @ wp + ice @ wi

    def selection(self, pred):
        """(screened top_k indices ascending by prediction, check indices, the
        band of ``deepen`` candidates below the top_k or None).  With a band,
        the first ``n_band`` check indices are drawn from it, the others from
        the rest; without one, all from the rest."""
        torch = _tm()
        order = torch.argsort(pred)
        top = order[:self.k]
        if self.deepen == 0:
            rest = order[self.k:]
            pick = torch.randperm(rest.numel(), generator=self.gen, device=pred.device)[:self.n_check]
            return top, rest[pick], None
        band, rest = order[self.k:self.k + self.deepen], order[self.k + self.deepen:]
        bp = torch.randperm(band.numel(), generator=self.gen, device=pred.device)[:self.n_band]
        rp = torch.randperm(rest.numel(), generator=self.gen, device=pred.device)[:self.n_check - self.n_band]
        return top, torch.cat([band[bp], rest[rp]]), band

    @staticmethod
    def _beats(best, others) -> float:
        """How much the best of ``others`` beats ``best``, relative to it (0 when it does not)."""
        if others.numel() == 0:
            return 0.0
        m = others.min()
        return float(((best - m) / m.abs().clamp(min=1e-9)).clamp(min=0.0).item())

    def __call__(self, Yn):
        torch = _tm()
        pred = self.predicted(Yn)
        top, chk, band = self.selection(pred)
        idx = torch.cat([top, chk])
        terms = self.dem_k.terms(Yn[idx].contiguous())
        exact = self.dem_k.total(terms)
        e_top, e_chk = exact[:self.k], exact[self.k:]
        best = e_top.min()
        nb = self.n_band if band is not None else 0
        band_miss = self._beats(best, e_chk[:nb])
        if nb:
            best = torch.minimum(best, e_chk[:nb].min())
        miss = self._beats(best, e_chk[nb:])
        self.rel_errs.append(miss)
        self.band_errs.append(band_miss)
        self.pred_errs.append(float(((pred[top] - e_top).abs() / e_top.abs().clamp(min=1e-9)).mean().item()))
        self.rollouts += idx.numel()
        if miss > self.max_rel_err:
            # screening misses better candidates than it keeps: the plain DEM scores all of them
            if self.dem_all is None:
                self.dem_all = DemScorer(self.scene, self.Q, self.w, **self.frame_kw)
            self.fallbacks += 1
            self.rollouts += self.Q
            all_terms = self.dem_all.terms(Yn)
            self._adapt(self._ext, all_terms[:, 4:7])
            return self.dem_all.total(all_terms)
        if self.n_check > nb and self.adapt_steps > 0:
            # the rest's check sample: drawn at random, unlike the top_k and the band
            self._adapt(self._ext[chk[nb:]], terms[self.k + nb:, 4:7])
        cost = torch.full_like(pred, float("inf"))
        cost[idx] = exact
        if band is not None and band_miss > self.max_rel_err:
            # the ranking misses near its cut: the DEM scores the whole band
            if self.dem_band is None:
                self.dem_band = DemScorer(self.scene, self.deepen, self.w, **self.frame_kw)
            self.deepened += 1
            self.rollouts += self.deepen
            cost[band] = self.dem_band(Yn[band].contiguous())
        return cost

    def close(self):
        """Release the DEM handles of the scorer's batches."""
        for d in (self.dem_k, self.dem_all, self.dem_band):
            if d is not None:
                d.batch.frame_step.close()

    def _adapt(self, ext, raw):
        """``adapt_steps`` Adam steps on rows ``ext`` with exact ice terms ``raw``."""
        if self.adapt_steps <= 0:
            return
        torch = _tm()
        net = self.sur.net
        m = int(ext.shape[0])
        B = min(256, m)
        if B < 16:
            return
        dev = ext.device
        if self._pat is None:
            self._pat = self.scene.patch.expand(256, -1, -1, -1).contiguous()
            self._grad = torch.empty((256, S.OUT_ROWS), dtype=torch.bfloat16, device=dev)
            self._loss = torch.empty(1, dtype=torch.float32, device=dev)
        tgt = self.sur.stats.forward(raw)
        for _ in range(self.adapt_steps):
            pick = torch.randperm(m, generator=self.gen, device=dev)[:B]
            out = net.forward(self._pat[:B], ext[pick].contiguous(), keep=True)
            sg_ops.mse(out, tgt[pick].contiguous(), S.N_OUT, self._grad[:B], self._loss)
            net.backward(self._grad[:B])
            net.adam_step(self.adapt_lr)

    def restore(self):
        """Put back the network (weights and Adam state) the scorer started from."""
        if self._base is not None:
            self.sur.net.load_state(self._base)


# ─── MBD (jax_mbd_planner.py:1314-1411) ─────────────────────────────────────
def mbd_plan(scorer, cfg: MBDConfig, device, seed: int = 0, Ybar_init=None):
    """Reverse diffusion in normalised (surge, yaw) action space; returns
    (Ybar (H, 2), per-step [mean cost, min cost])."""
    torch = _tm()
    H, Ns = cfg.horizon, cfg.n_sample
    if Ybar_init is None:
        Ybar = torch.zeros((H, 2), dtype=torch.float32, device=device)
        Ybar[:, 0] = cfg.init_surge_bias
    else:
        Ybar = torch.clamp(torch.as_tensor(Ybar_init, dtype=torch.float32, device=device), -1.0, 1.0)
    if cfg.n_diffuse <= 1:
        return Ybar, []
    betas = torch.linspace(cfg.beta0, cfg.betaT, cfg.n_diffuse, dtype=torch.float32, device=device)
    alphas = 1.0 - betas
    alphas_bar = torch.cumprod(alphas, 0)
    sigmas = torch.sqrt(1.0 - alphas_bar)
    gen = torch.Generator(device=device).manual_seed(seed)
    metrics = []
    i = cfg.n_diffuse - 1
    for _ in range(cfg.n_diffuse - 1):
        Yi = Ybar * torch.sqrt(alphas_bar[i])
        eps = torch.randn((Ns, H, 2), generator=gen, dtype=torch.float32, device=device)
        Y0s = torch.clamp(eps * sigmas[i] + Ybar, -1.0, 1.0)
        costs = scorer(Y0s).float()
        rews = -costs
        logp0 = (rews - rews.max()) / cfg.temperature
        weights = torch.softmax(logp0, 0)
        Ybar_new = torch.einsum("n,nij->ij", weights, Y0s)
        score = 1.0 / (1.0 - alphas_bar[i]) * (-Yi + torch.sqrt(alphas_bar[i]) * Ybar_new)
        Yim1 = 1.0 / torch.sqrt(alphas[i]) * (Yi + (1.0 - alphas_bar[i]) * score)
        i_prev = max(i - 1, 0)
        Ybar = torch.clamp(Yim1 / torch.sqrt(alphas_bar[i_prev]), -1.0, 1.0)
        fin = costs[torch.isfinite(costs)]  # a screened step leaves the unchecked candidates at +inf
        metrics.append((fin.mean(), fin.min()))
        i -= 1
    return Ybar, [(float(a), float(b)) for a, b in metrics]


def plan_cost(scene: PlanScene, Ybar, dem: DemScorer) -> float:
    """The DEM cost of executing a plan (every system of ``dem`` runs it; the first is read)."""
    Y = Ybar.unsqueeze(0).expand(dem.Q, -1, -1).contiguous()
    return float(dem(Y)[0].item())


# ─── training data: DEM rollouts from the batched-rollout generator ─────────
def sample_starts(field, n: int, rng, horizon: int = 64, clearance: float = 2.0):
    """Start poses in open water among the floes: heading along the field's
    track +- 0.3 rad, no element within the hull box plus ``clearance``, and
    ice within reach of the bow (a window of at least 20 elements)."""
    cents = np.asarray(field.centroids, np.float64)
    x0, x1, y0, y1 = field.domain
    L, B = field.ship_length, field.ship_beam
    R = reach_radius(field, horizon, field.dt)
    from scipy.spatial import cKDTree
    tree = cKDTree(cents)
    out = []
    tries = 0
    base = float(field.trajectory[0][2])
    while len(out) < n and tries < 200000:
        tries += 1
        x, y = rng.uniform(x0 + 20, x1 - 20), rng.uniform(y0 + 20, y1 - 20)
        psi = base + rng.uniform(-0.3, 0.3)
        c, s = math.cos(psi), math.sin(psi)
        near = tree.query_ball_point([x, y], 0.5 * math.hypot(L, B) + clearance + 3.0)
        ok = True
        for k in near:
            dx, dy = cents[k, 0] - x, cents[k, 1] - y
            bx, by = c * dx + s * dy, -s * dx + c * dy
            if abs(bx) < 0.5 * L + clearance and abs(by) < 0.5 * B + clearance:
                ok = False
                break
        if not ok:
            continue
        if len(tree.query_ball_point([x, y], R)) < 20:
            continue
        out.append(np.array([x, y, psi]))
    return out


def element_radii(field) -> np.ndarray:
    """Largest centroid-to-vertex distance of each element's polygon."""
    cents = np.asarray(field.centroids, np.float64)
    return np.array([float(np.max(np.hypot(*(np.asarray(p, np.float64) - c).T))) for p, c in
                     zip(field.polygons, cents)])


def channel_starts(field, n: int, rng, horizon: int = 64, clearance: float = 2.0, channel: float = 100.0,
                   radii=None):
    """Mid-transit start poses inside the pack, each with the elements its
    passage has cleared: the ship at a uniform position whose reach stays
    inside the field's ice, heading along the field's track +- 0.3 rad, with
    every element that overlaps the hull box plus ``clearance`` or the
    ``channel`` metres of beam-wide lane behind the stern removed.  Returns
    ``[(eta, removed_indices)]``; windows hold the full pack density."""
    cents = np.asarray(field.centroids, np.float64)
    radii = element_radii(field) if radii is None else np.asarray(radii, np.float64)
    L, B = field.ship_length, field.ship_beam
    R = reach_radius(field, horizon, field.dt)
    lo, hi = cents.min(0) + R + 10.0, cents.max(0) - R - 10.0
    if np.any(hi <= lo):
        raise ValueError("the field's ice is smaller than one planning window")
    from scipy.spatial import cKDTree
    tree = cKDTree(cents)
    rmax = float(radii.max())
    base = float(field.trajectory[0][2])
    out = []
    for _ in range(n):
        x, y = rng.uniform(lo[0], hi[0]), rng.uniform(lo[1], hi[1])
        psi = base + rng.uniform(-0.3, 0.3)
        c, s = math.cos(psi), math.sin(psi)
        near = np.asarray(tree.query_ball_point([x, y], 0.5 * L + channel + B + clearance + rmax), np.int64)
        dx, dy = cents[near, 0] - x, cents[near, 1] - y
        bx, by = c * dx + s * dy, -s * dx + c * dy
        r = radii[near] + clearance
        gone = (bx < 0.5 * L + r) & (bx > -0.5 * L - channel - r) & (np.abs(by) < 0.5 * B + r)
        out.append((np.array([x, y, psi]), near[gone]))
    return out


def sample_training_controls(rng, Q: int, H: int, device):
    """(Q, H, 2) normalised controls: half Gaussian around the surge bias (sigma
    0.3 of the maxima, the batched-rollout generator's spread), half uniform."""
    torch = _tm()
    g = rng.normal(0.0, 0.3, (Q, H, 2))
    g[..., 0] += MBDConfig.init_surge_bias
    u = rng.uniform(-1.0, 1.0, (Q, H, 2))
    pick = rng.random(Q) < 0.5
    y = np.where(pick[:, None, None], g, u)
    return torch.as_tensor(np.clip(y, -1.0, 1.0), dtype=torch.float32, device=device)


@dataclass
class Dataset:
    patches: object     # (S, 64, 64, 1) bf16, normalised
    start_of: object    # (N,) int32 start index of each sample
    extra: object       # (N, 6 + 3H) fp32 (``features``)
    raw: object         # (N, 3) float64 ice terms [KE, impulse, bonds]
    planner: object     # (N, 4) float64 planner components of the DEM paths
    patch_stats: tuple
    seconds: float = 0.0


def scene_starts(field, kind: str, n: int, rng, horizon: int = 64):
    """``n`` plan starts as ``[(eta, removed)]``: ``"open"`` water among the
    floes (nothing removed) or mid-transit ``"channel"`` starts in the pack."""
    if kind == "open":
        return [(e, None) for e in sample_starts(field, n, rng, horizon)]
    if kind == "channel":
        return channel_starts(field, n, rng, horizon)
    raise ValueError(f"unknown scene kind {kind!r}")


def generate_dataset(field, n_starts: int, per_start: int, horizon: int = 64, seed: int = 0, device="cuda",
                     patch_stats=None, weights: Optional[CostWeights] = None, scenes: str = "open",
                     **frame_kw) -> Dataset:
    """``n_starts`` x ``per_start`` DEM rollouts (one batched launch per start)
    from ``scenes`` starts (``scene_starts``)."""
    torch = _tm()
    from .config import get_default_simulation_config
    from .state import build_static_arrays, ship_dynamics_arrays
    t0 = time.time()
    rng = np.random.default_rng(seed)
    cfg = get_default_simulation_config()
    static = build_static_arrays(field.polygons, field.centroids, field.bonds, field.thicknesses, field.parent_ids,
                                 cfg, DEFAULT_MATERIAL, 0.05)
    sd = ship_dynamics_arrays(field.ship_props, cfg, field.ship_length, field.ship_beam, field.hull_local)
    starts = scene_starts(field, scenes, n_starts, rng, horizon)
    raw_patches, extras, raws, plans, start_of = [], [], [], [], []
    w = weights or CostWeights()
    for si, (e0, rem) in enumerate(starts):
        nu0 = np.array([rng.uniform(1.0, 3.0), 0.0, 0.0])
        sc = make_scene(field, e0, nu0, horizon, device=device, static=static, ship_dyn=sd, removed=rem)
        c0 = (COSTMAP_CELLS - PATCH_CELLS) // 2
        raw_patches.append(sc.costmap.grid[c0:c0 + PATCH_CELLS, c0:c0 + PATCH_CELLS].clone())
        Yn = sample_training_controls(rng, per_start, horizon, sc.device)
        dem = DemScorer(sc, per_start, w, **frame_kw)
        terms = dem.terms(Yn)
        extras.append(features(sc, Yn, *rigid_path(sc, Yn)[1:]))
        plans.append(terms[:, :4].clone())
        raws.append(terms[:, 4:7].clone())
        start_of.append(torch.full((per_start,), si, dtype=torch.int32, device=sc.device))
        dem.batch.frame_step.close()
        del dem
    P = torch.stack(raw_patches)
    if patch_stats is None:
        patch_stats = (float(P.mean().item()), float(P.std().item()) or 1.0)
    Pn = sg_ops.to_bf16(((P - patch_stats[0]) / patch_stats[1]).contiguous()).view(len(starts), PATCH_CELLS,
                                                                                    PATCH_CELLS, 1)
    torch.cuda.synchronize()
    return Dataset(Pn, torch.cat(start_of), torch.cat(extras), torch.cat(raws), torch.cat(plans), patch_stats,
                   time.time() - t0)


def mirror_rows(patches, extra):
    """The mirror image of training rows about the ship's start axis, in place:
    the patch flipped left-right (x about the ship), sway velocity, yaw rate,
    cos(heading) and every yaw control negated.  The hull is symmetric, so the
    mirrored scene has the same ice terms, and the mirrored path meets the
    same costmap values and sweeps the same ice; the patch is centred on the
    ship."""
    torch = _tm()
    H = (int(extra.shape[1]) - S.N_SHIP - S.N_SWEEP) // S.N_STEP
    patches.copy_(torch.flip(patches, dims=[2]))
    extra[:, 1] = -extra[:, 1]
    extra[:, 2] = -extra[:, 2]
    extra[:, 3] = -extra[:, 3]
    extra[:, S.N_SHIP + 1:S.N_SHIP + 2 * H:2] = -extra[:, S.N_SHIP + 1:S.N_SHIP + 2 * H:2]


def train_surrogate(data: Dataset, horizon: int = 64, epochs: int = 8, batch: int = 256, lr: float = 1e-3,
                    seed: int = 0, holdout: float = 0.1, device="cuda", mirror: bool = True):
    """Adam on fp32 master weights, BF16 tensor-core forward and backward.  Whole
    starts are held out; half of every batch is mirrored (``mirror_rows``); the
    weights of the epoch with the lowest held-out loss are kept.  Returns
    (Surrogate, {"train_loss", "holdout_loss" (per epoch), "best_epoch",
    "seconds", "steps", ...})."""
    torch = _tm()
    t0 = time.time()
    dev = torch.device(device)
    raw = data.raw
    # target statistics on the log1p transform
    sc = torch.tensor(TARGET_SCALE, dtype=torch.float64, device=dev)
    t = torch.log1p(torch.clamp(raw, min=0.0) / sc)
    stats = TargetStats(t.mean(0).cpu().numpy(), np.maximum(t.std(0).cpu().numpy(), 1e-6))
    tgt = stats.forward(raw).contiguous()
    rng = np.random.default_rng(seed)
    # hold out whole starts (unseen ice)
    n_starts = int(data.patches.shape[0])
    hold = set(rng.choice(n_starts, max(1, int(round(holdout * n_starts))), replace=False).tolist())
    so = data.start_of.cpu().numpy()
    train_idx = np.nonzero(~np.isin(so, list(hold)))[0]
    hold_idx = np.nonzero(np.isin(so, list(hold)))[0]
    net = S.SurrogateNet(horizon=horizon, device=dev, seed=seed)
    sur = Surrogate(net, stats, data.patch_stats)
    Bz = batch
    ext_b = torch.empty((Bz, data.extra.shape[1]), dtype=torch.float32, device=dev)
    tgt_b = torch.empty((Bz, S.N_OUT), dtype=torch.float32, device=dev)
    pat_b = torch.empty((Bz, PATCH_CELLS, PATCH_CELLS, 1), dtype=torch.bfloat16, device=dev)
    grad = torch.empty((Bz, S.OUT_ROWS), dtype=torch.bfloat16, device=dev)
    loss = torch.empty(1, dtype=torch.float32, device=dev)
    half = Bz // 2
    steps = 0
    losses, hlosses = [], []
    best, best_ep, snap = float("inf"), -1, None
    for ep in range(epochs):
        perm = rng.permutation(train_idx)
        for b0 in range(0, len(perm) - Bz + 1, Bz):
            idx = torch.as_tensor(perm[b0:b0 + Bz], dtype=torch.int32, device=dev)
            sidx = data.start_of[idx.long()]
            sg_ops.gather_rows(data.extra, idx, ext_b)
            sg_ops.gather_rows(tgt, idx, tgt_b)
            sg_ops.gather_rows(data.patches.view(n_starts, -1), sidx, pat_b.view(Bz, -1))
            if mirror:
                mirror_rows(pat_b[:half], ext_b[:half])
            out = net.forward(pat_b, ext_b, keep=True)
            sg_ops.mse(out, tgt_b, S.N_OUT, grad, loss)
            net.backward(grad)
            net.adam_step(lr * (0.5 * (1 + math.cos(math.pi * ep / max(epochs, 1)))))
            steps += 1
        losses.append(float(loss.item()))
        hl = holdout_error(sur, data, hold_idx, tgt) if len(hold_idx) else float("nan")
        hlosses.append(hl)
        if hl < best:
            best, best_ep = hl, ep
            snap = [(p.p.clone(), p.b.clone()) for p in net.params()]
    if snap is not None:
        for layer, (pw, pb) in zip(net.params(), snap):
            layer.p.copy_(pw)
            layer.b.copy_(pb)
            sg_ops.to_bf16(layer.p, out=layer.w)
            sg_ops.transpose(layer.w, out=layer.wt)
    sg_ops.error_flag(dev).check()
    return sur, {"train_loss": losses, "holdout_loss": hlosses, "best_epoch": best_ep,
                 "holdout_best": best, "seconds": time.time() - t0, "steps": steps,
                 "train_samples": int(len(train_idx)), "holdout_samples": int(len(hold_idx))}


def within_scene_rank_corr(data: Dataset) -> dict:
    """Mean over the dataset's starts of the Spearman rank correlation, among
    one start's candidates, between each network input summary and each ice
    term: the sweep features (``SWEEP_SCALE`` order) and the sum of the path's
    log costmap values, against [KE, impulse, bonds].  How well an input can
    rank the candidates of one scene, which is what screening needs."""
    from scipy.stats import rankdata
    extra = data.extra.detach().cpu().numpy().astype(np.float64)
    raw = data.raw.detach().cpu().numpy().astype(np.float64)
    so = data.start_of.detach().cpu().numpy()
    H = (extra.shape[1] - S.N_SHIP - S.N_SWEEP) // S.N_STEP
    names = ["elements_hit", "mass_hit", "ke_proxy", "momentum_proxy", "mass_early", "ke_normal_proxy",
             "bonds_cut", "bonds_inside", "path_costmap"]
    path = extra[:, S.N_SHIP + 2 * H:S.N_SHIP + 3 * H].sum(1, keepdims=True)
    feats = np.concatenate([extra[:, S.N_SHIP + 3 * H:], path], 1)
    acc = np.zeros((len(names), 3))
    cnt = np.zeros((len(names), 3))
    for st in np.unique(so):
        m = so == st
        for j in range(len(names)):
            fr = rankdata(feats[m, j])
            for k in range(3):
                tr = rankdata(raw[m, k])
                if np.std(fr) > 0 and np.std(tr) > 0:
                    acc[j, k] += np.corrcoef(fr, tr)[0, 1]
                    cnt[j, k] += 1
    mean = np.where(cnt > 0, acc / np.maximum(cnt, 1), np.nan)
    return {nm: {"ke": float(mean[j, 0]), "impulse": float(mean[j, 1]), "bonds": float(mean[j, 2])}
            for j, nm in enumerate(names)}


def holdout_error(sur: Surrogate, data: Dataset, idx, tgt) -> float:
    """Mean squared error of the standardised targets on held-out samples."""
    torch = _tm()
    dev = data.extra.device
    errs = []
    B = 1024
    for b0 in range(0, len(idx), B):
        ii = torch.as_tensor(idx[b0:b0 + B], dtype=torch.int32, device=dev)
        n = int(ii.shape[0])
        ext = torch.empty((n, data.extra.shape[1]), dtype=torch.float32, device=dev)
        sg_ops.gather_rows(data.extra, ii, ext)
        pat = torch.empty((n, PATCH_CELLS, PATCH_CELLS, 1), dtype=torch.bfloat16, device=dev)
        sg_ops.gather_rows(data.patches.view(data.patches.shape[0], -1), data.start_of[ii.long()], pat.view(n, -1))
        out = sur.net.forward(pat, ext)
        errs.append(((out[:, :S.N_OUT] - tgt[ii.long()]) ** 2).mean().item() * n)
    return float(sum(errs) / len(idx))
