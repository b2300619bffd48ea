"""Scenario plumbing shared by the CPU oracle tests and the GPU parity tests.

Every scenario is rebuilt from the committed golden files: the static data
and vessel matrices are the ones the reference's own builders produced, and
the initial states/setpoints are the ones the golden run used.
"""
from __future__ import annotations

import math
from types import SimpleNamespace

import numpy as np

from oracle.dem_oracle import OParams, OShip, OState, Oracle, params_from_config

STATIC_FIELDS = ("local_polys_padded", "poly_mask", "poly_n_verts", "masses", "inertia", "radii",
                 "areas", "thicknesses", "bond_i", "bond_j", "rest_lengths", "bond_strengths",
                 "bond_areas", "sigma_bar_bond", "initial_floe_of", "k_n", "k_s")
SHIPDYN_FIELDS = ("M3inv", "D3", "mass", "Izz", "Kp", "Kd", "Ki", "B_pinv", "n_max", "ship_hull_local")

# material of the small three-floe workload (rho 900, 0.5 MPa) and its dilation
SMALL_FLEX = 0.5e6

B_THRUST = np.array([[0, 0, 0, 0, 1, 1], [1, 1, 1, 1, 0, 0], [30, 22, -22, -30, -8, 8]], float) \
    @ np.diag([3.2, 3.2, 3.2, 3.2, 31.2, 31.2])


def default_cfg():
    from mbd_icenav_b200.config import SimulationConfig
    return SimulationConfig()


def static_from_golden(g, prefix):
    d = {}
    for k in STATIC_FIELDS:
        v = g[f"{prefix}_static_{k}"]
        d[k] = float(v) if k in ("k_n", "k_s") else np.asarray(v)
    d["pair_i"] = d["pair_j"] = None
    return SimpleNamespace(**d)


def shipdyn_from_golden(g, prefix):
    d = {}
    for k in SHIPDYN_FIELDS:
        v = g[f"{prefix}_shipdyn_{k}"]
        d[k] = float(v) if k in ("mass", "Izz") else np.asarray(v)
    return SimpleNamespace(**d)


SCENARIOS = {
    # prefix: (ship_length, ship_beam, n_ice_steps, dt, dt_ice, use_auto, flexural base)
    "hex": (15.0, 5.0, 1, 0.05, 0.05, False, 0.3e6),
    "small": (60.0, 12.0, 10, 0.05, 0.005, False, SMALL_FLEX),
    "window": (60.0, 12.0, 10, 0.05, 0.005, True, 0.3e6),
}


def scenario_params(prefix, cfg=None) -> OParams:
    L, B, k, dt, dti, auto, flex = SCENARIOS[prefix]
    return params_from_config(cfg or default_cfg(), L, B, k, dt, dti, auto, 1.0,
                              flexural_strength_base=flex)


def initial_state(g, prefix, dtype=np.float64):
    static = static_from_golden(g, prefix)
    n = static.masses.shape[0]
    nb = static.bond_i.shape[0]
    nf = int(static.initial_floe_of.max()) + 1
    cents = np.asarray(g[f"{prefix}_centroids"], np.float64)
    st = OState(positions=cents.astype(dtype), velocities=np.zeros((n, 2), dtype),
                rotations=np.zeros(n, dtype), angular_vels=np.zeros(n, dtype),
                submergence=np.zeros(n, dtype), bond_intact=np.ones(nb, bool),
                bond_damage=np.zeros(nb, dtype), bond_delta_m_0=np.zeros(nb, dtype),
                bond_delta_m_max=np.zeros(nb, dtype), bond_delta_s=np.zeros(nb, dtype),
                elem_active=np.zeros(n, bool), dpdem_floe_eligible=np.zeros(nf, bool))
    if prefix == "hex":
        eta0 = np.array([-25.0, 0.0, 0.0])
    elif prefix == "small":
        eta0 = np.asarray(g["small_ship0"], np.float64)
    else:
        eta0 = np.asarray(g["window_ship0"], np.float64)
        st = st._replace(velocities=np.asarray(g["window_vel0"], np.float64).astype(dtype),
                         elem_active=np.ones(n, bool), dpdem_floe_eligible=np.ones(nf, bool))
    ship = OShip(eta=eta0.astype(dtype), nu=np.zeros(3, dtype), n_actual=np.zeros(6, dtype),
                 e_int=np.zeros(3, dtype))
    return st, ship


def frame_inputs(g, prefix, f):
    """(setpoint, setpoint_next, v_water (n,2), v_water_ship (2,)) for frame f."""
    static = static_from_golden(g, prefix)
    n = static.masses.shape[0]
    if prefix == "hex":
        tr = np.asarray(g["hex_traj"], np.float64)
        return tr[f], tr[f + 1], np.zeros((n, 2)), np.zeros(2)
    if prefix == "small":
        sp = np.asarray(g["small_setpoints"], np.float64)
        return sp[f, :3], sp[f, 3:], np.zeros((n, 2)), np.zeros(2)
    sp = np.asarray(g["window_sp"], np.float64)
    return sp[f], sp[f + 1], np.asarray(g["window_vw"], np.float64), np.array([0.05, 0.02])


def make_oracle(g, prefix, dtype=np.float64, pair_mode="all") -> Oracle:
    return Oracle(static_from_golden(g, prefix), shipdyn_from_golden(g, prefix),
                  scenario_params(prefix), B_THRUST, dtype=dtype, pair_mode=pair_mode)


def fn_static(g):
    return static_from_golden(g, "fn")


def rel_err(a, b, floor=None):
    """max |a-b| / max(|b|max, floor): a norm-wise relative error."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = np.max(np.abs(b)) if b.size else 0.0
    if floor is not None:
        scale = max(scale, floor)
    if scale == 0.0:
        return float(np.max(np.abs(a - b))) if a.size else 0.0
    return float(np.max(np.abs(a - b)) / scale)


# ── GPU-side construction from the same golden data ─────────────────────────

def gpu_frame_step(g, prefix, torch_dtype, **kw):
    """FrameStep (libdem_b200) bound to a golden scenario's static data."""
    import torch
    from mbd_icenav_b200 import sim
    from mbd_icenav_b200.config import IceMaterial
    L, B, k, dt, dti, auto, flex = SCENARIOS[prefix]
    dev = torch.device("cuda", 0)
    st = static_from_golden(g, prefix)
    sd = shipdyn_from_golden(g, prefix)
    mat = IceMaterial(flexural_strength_base=flex)
    return sim.make_frame_step(st, default_cfg(), sd, L, B, k, dt, dti, auto, B_THRUST, 1.0,
                               material=mat, device=dev, dtype=torch_dtype, **kw)


def to_gpu_state(st, ship, torch_dtype):
    import torch
    from mbd_icenav_b200.state import IceState, ShipState
    dev = torch.device("cuda", 0)
    f = lambda a: torch.as_tensor(np.asarray(a, np.float64)).to(dev, torch_dtype)
    b = lambda a: torch.as_tensor(np.asarray(a, bool)).to(dev)
    ice = IceState(positions=f(st.positions), velocities=f(st.velocities), rotations=f(st.rotations),
                   angular_vels=f(st.angular_vels), submergence=f(st.submergence),
                   bond_intact=b(st.bond_intact), bond_damage=f(st.bond_damage),
                   bond_delta_m_0=f(st.bond_delta_m_0), bond_delta_m_max=f(st.bond_delta_m_max),
                   bond_delta_s=f(st.bond_delta_s), elem_active=b(st.elem_active),
                   dpdem_floe_eligible=b(st.dpdem_floe_eligible))
    sh = ShipState(eta=f(ship.eta), nu=f(ship.nu), n_actual=f(ship.n_actual), e_int=f(ship.e_int))
    return ice, sh


def to_np_state(st, ship):
    ice = OState(*[t.detach().cpu().numpy() for t in st])
    sh = OShip(*[t.detach().cpu().numpy() for t in ship])
    return ice, sh
