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


# ── per-element step comparison (fp32 parity at the stated tolerance) ───────

STEP_REL = 1e-5  # per-step relative tolerance in fp32 (positions, velocities, forces, state)
STEP_ULPS = 4    # absolute floor: this many fp32 rounding units of the quantity itself


def ulp32(x):
    """fp32 rounding unit (spacing) of |x|, as float64."""
    return np.spacing(np.abs(np.asarray(x, np.float64)).astype(np.float32)).astype(np.float64)


def step_ratio(got, want, before, rel=STEP_REL, ulps=STEP_ULPS, want64=None):
    """Per entry (per row for (m, 2) arrays): |got - want| / (rel |want - before| +
    ulps ulp32(max(|want|, |before|)) + 2 |want - want64|), the error against the
    step's own change with a floor at fp32 rounding of the values.  With
    ``want64`` (the same step in float64 from the same input), the allowance
    also holds twice the fp32 reference's own error: where the fp32 reference is
    less accurate than ``rel`` of the change (a quantity formed by
    cancellation, such as a torque whose terms nearly balance), the result must
    be at least about as accurate as it.  Returns the array of ratios (<= 1
    passes) — 0 where both agree exactly."""
    g = np.asarray(got, np.float64)
    w = np.asarray(want, np.float64)
    b = np.asarray(before, np.float64)
    mag = np.maximum(np.abs(w), np.abs(b))
    if g.ndim == 2:
        err = np.sqrt(((g - w) ** 2).sum(1))
        change = np.sqrt(((w - b) ** 2).sum(1))
        floor = ulps * ulp32(mag.max(1))
    else:
        err = np.abs(g - w)
        change = np.abs(w - b)
        floor = ulps * ulp32(mag)
    if want64 is not None:
        w64 = np.asarray(want64, np.float64)
        own = np.sqrt(((w - w64) ** 2).sum(1)) if g.ndim == 2 else np.abs(w - w64)
        floor = floor + 2.0 * np.where(np.isfinite(own), own, 0.0)
    both_nan = np.isnan(g) & np.isnan(w)
    if g.ndim == 2:
        both_nan = both_nan.all(1)
    err = np.where(both_nan, 0.0, err)
    return err / (rel * change + floor)


def assert_step_close(name, got, want, before, rel=STEP_REL, ulps=STEP_ULPS, want64=None):
    """Every entry within ``rel`` of its own step change (floor: fp32 rounding, and
    with ``want64`` twice the fp32 reference's own error against float64)."""
    r = step_ratio(got, want, before, rel, ulps, want64)
    if r.size and not (np.nanmax(r) <= 1.0):
        i = int(np.nanargmax(r))
        raise AssertionError(f"{name}: entry {i} off by {np.nanmax(r):.3g}x the tolerance "
                             f"(got {np.asarray(got)[i]}, want {np.asarray(want)[i]}, "
                             f"before {np.asarray(before)[i]}); {int((r > 1).sum())} entries out")
    return float(np.nanmax(r)) if r.size else 0.0


ICE_FLOAT_FIELDS = ("positions", "velocities", "rotations", "angular_vels", "submergence", "bond_damage",
                    "bond_delta_m_0", "bond_delta_m_max", "bond_delta_s")
ICE_MASK_FIELDS = ("bond_intact", "elem_active", "dpdem_floe_eligible")
SHIP_FIELDS = ("eta", "nu", "n_actual", "e_int")


def assert_frame_matches(ice, ship, o_ice, o_ship, in_ice, in_ship, diag=None, o_diag=None, where="",
                         o_ice64=None, o_ship64=None):
    """One frame from identical inputs, GPU vs oracle: every IceState and
    ShipState field (masks bit-equal; floats per entry within the step
    tolerance, see ``step_ratio``; ``o_ice64`` / ``o_ship64`` are the float64
    oracle's frame from the same input), and the diagnostics (contact mask,
    force magnitudes, ship force).  Returns the worst ratio per field."""
    worst = {}
    for f in ICE_MASK_FIELDS:
        np.testing.assert_array_equal(getattr(ice, f), getattr(o_ice, f), err_msg=f"{f} {where}")
    for f in ICE_FLOAT_FIELDS:
        w64 = None if o_ice64 is None else getattr(o_ice64, f)
        worst[f] = assert_step_close(f"{f} {where}", getattr(ice, f), getattr(o_ice, f), getattr(in_ice, f),
                                     want64=w64)
    for f in SHIP_FIELDS:
        w64 = None if o_ship64 is None else getattr(o_ship64, f)
        worst[f] = assert_step_close(f"ship {f} {where}", getattr(ship, f), getattr(o_ship, f),
                                     getattr(in_ship, f), want64=w64)
    if diag is not None:
        gp = diag["pen_max"].detach().cpu().numpy()
        np.testing.assert_array_equal(gp > 0, o_diag["pen_max"] > 0, err_msg=f"contact mask {where}")
        z = np.zeros_like(o_diag["force_mag"])
        worst["force_mag"] = assert_step_close(f"force_mag {where}", diag["force_mag"].detach().cpu().numpy(),
                                               o_diag["force_mag"], z)
        worst["pen_max"] = assert_step_close(f"pen_max {where}", gp, o_diag["pen_max"], np.zeros_like(gp))
        worst["F_ice_on_ship"] = assert_step_close(f"F_ice_on_ship {where}",
                                                   diag["F_ice_on_ship"].detach().cpu().numpy()[None],
                                                   np.asarray(o_diag["F_ice_on_ship"])[None],
                                                   np.zeros((1, 2)))
    return worst


def contact_sets_match(sets, raw, o_sets, active, where=""):
    """GPU contact sets (per substep, recorded from active elements) against
    the oracle's (all pairs): equal on the pairs with an active end, and every
    pair of two active elements recorded from both ends."""
    assert len(sets) == len(o_sets), (len(sets), len(o_sets))
    total = 0
    for s, (g, o, r) in enumerate(zip(sets, o_sets, raw)):
        o_act = {(i, j) for i, j in o if active[i] or active[j]}
        missing, extra = o_act - g, g - o_act
        assert not missing and not extra, (f"substep {s} {where}: {len(missing)} contacts missing "
                                           f"(e.g. {sorted(missing)[:3]}), {len(extra)} extra "
                                           f"(e.g. {sorted(extra)[:3]})")
        both = {(i, j) for i, j in g if active[i] and active[j]}
        seen = set(map(tuple, r.tolist()))
        for i, j in both:
            assert (i, j) in seen and (j, i) in seen, f"substep {s} {where}: pair {(i, j)} recorded from one end"
        assert len(r) == len(g) + len(both), f"substep {s} {where}: repeated records"
        total += len(g)
    return total
