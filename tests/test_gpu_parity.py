"""GPU parity: libdem_b200 (through its C ABI) vs the reference's outputs and the oracle.

* float64 free runs vs the golden vectors (the reference's own code, every
  recorded field) and vs the float64 oracle (every IceState / ShipState field);
* float32 single frames from identical input states vs the float32 oracle:
  every float field per entry within 1e-5 of its own change over the frame
  (floor: fp32 rounding of the value, and twice the fp32 oracle's own error
  against the float64 oracle from the same input), masks and the contact mask
  bit-equal;
* the ice-ice contact set of every substep bit-equal to the oracle's
  (overlap > 0 and distance > 1e-6, jax_simulation.py:127-131);
* scan == frame loop and persistent == phased launches, bit for bit;
* float32 drift over 1,000 substeps against the float64 oracle.
"""
import numpy as np
import pytest

from helpers import (ICE_FLOAT_FIELDS, ICE_MASK_FIELDS, SHIP_FIELDS, assert_frame_matches, contact_sets_match,
                     frame_inputs, gpu_frame_step, initial_state, make_oracle, rel_err, to_gpu_state, to_np_state)

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

# golden key -> (state, field) of the reference's recorded histories
GOLDEN_FIELDS = {"pos": ("ice", "positions"), "vel": ("ice", "velocities"), "rot": ("ice", "rotations"),
                 "avel": ("ice", "angular_vels"), "sub": ("ice", "submergence"), "damage": ("ice", "bond_damage"),
                 "dm0": ("ice", "bond_delta_m_0"), "dmmax": ("ice", "bond_delta_m_max"),
                 "ds": ("ice", "bond_delta_s"), "eta": ("ship", "eta"), "nu": ("ship", "nu"),
                 "n_actual": ("ship", "n_actual")}
F64_TOL = 1e-9  # norm-wise relative, float64 free runs (measured ~1e-15)


def _frame(fs, st, sh, g, prefix, f, dtype):
    sp, spn, vw, vws = frame_inputs(g, prefix, f)
    d = torch.device("cuda", 0)
    t = lambda a: torch.as_tensor(np.asarray(a, np.float64)).to(d, dtype)
    return fs(st, sh, t(sp), t(spn), t(vw), st.dpdem_floe_eligible, t(vws))


@pytest.mark.parametrize("prefix", ["hex", "small", "window"])
def test_f64_free_run_matches_reference(prefix, golden64):
    """Free-running float64 GPU frames vs the reference's recorded run (every
    recorded field) and vs the float64 oracle run alongside (every field,
    the integral error e_int included)."""
    g = golden64
    fs = gpu_frame_step(g, prefix, torch.float64)
    o = make_oracle(g, prefix, np.float64, pair_mode="grid")
    o_st, o_sh = initial_state(g, prefix, np.float64)
    st, sh = to_gpu_state(o_st, o_sh, torch.float64)
    n_frames = g[f"{prefix}_pos"].shape[0]
    worst = {}
    for f in range(n_frames):
        sp, spn, vw, vws = frame_inputs(g, prefix, f)
        o_st, o_sh, _ = o.frame_step(o_st, o_sh, sp, spn, vw, o_st.dpdem_floe_eligible, vws)
        st, sh, diag = _frame(fs, st, sh, g, prefix, f, torch.float64)
        ice, ship = to_np_state(st, sh)
        for key, (kind, name) in GOLDEN_FIELDS.items():
            if f"{prefix}_{key}" not in g.files:
                continue
            got = getattr(ice if kind == "ice" else ship, name)
            e = rel_err(got, g[f"{prefix}_{key}"][f], 1.0)
            worst[key] = max(worst.get(key, 0.0), e)
            assert e < F64_TOL, (f, key, e)
        for name in ICE_FLOAT_FIELDS:
            assert rel_err(getattr(ice, name), getattr(o_st, name), 1.0) < F64_TOL, (f, name)
        for name in SHIP_FIELDS:
            assert rel_err(getattr(ship, name), getattr(o_sh, name), 1.0) < F64_TOL, (f, name)
        for name in ICE_MASK_FIELDS:
            np.testing.assert_array_equal(getattr(ice, name), getattr(o_st, name), err_msg=f"{name} frame {f}")
        np.testing.assert_array_equal(ice.bond_intact, g[f"{prefix}_intact"][f], err_msg=f"frame {f}")
        np.testing.assert_array_equal(ice.elem_active, g[f"{prefix}_active"][f])
        np.testing.assert_array_equal(ice.dpdem_floe_eligible, g[f"{prefix}_elig"][f])
        np.testing.assert_array_equal(diag["pen_max"].cpu().numpy() > 0, g[f"{prefix}_pen"][f] > 0)
        assert rel_err(diag["force_mag"].cpu().numpy(), g[f"{prefix}_fmag"][f], 1.0) < F64_TOL
        assert rel_err(diag["F_ice_on_ship"].cpu().numpy(), g[f"{prefix}_F"][f], 1.0) < F64_TOL
        assert rel_err(diag["J_cumul_incr"].cpu().numpy(), g[f"{prefix}_J"][f], 1.0) < F64_TOL
    print(prefix, "worst norm-wise relative error per field:", {k: f"{v:.2e}" for k, v in worst.items()})
    fs.close()


@pytest.mark.parametrize("prefix", ["hex", "small", "window"])
def test_f32_single_frames_match_oracle(prefix, golden32):
    """Same fp32 input state -> one frame on GPU and in the fp32 oracle; every
    field per entry within 1e-5 of its own change over the frame, or, where the
    fp32 oracle itself is farther than that from the float64 oracle (a sum
    that cancels, such as a torque whose normal-force terms balance), within
    twice the fp32 oracle's own error."""
    g = golden32
    fs = gpu_frame_step(g, prefix, torch.float32)
    o = make_oracle(g, prefix, np.float32, pair_mode="grid")
    o64 = make_oracle(g, prefix, np.float64, pair_mode="grid")  # the fp32 reference's own error
    st, sh = initial_state(g, prefix, np.float32)
    n_frames = g[f"{prefix}_pos"].shape[0]
    checked = 0
    worst = {}
    for f in range(n_frames):
        sp, spn, vw, vws = frame_inputs(g, prefix, f)
        c = lambda a: np.asarray(a, np.float64).astype(np.float32)
        o_st, o_sh, o_diag = o.frame_step(st, sh, c(sp), c(spn), c(vw), st.dpdem_floe_eligible, c(vws))
        if prefix != "small" or f % 5 == 0 or (o_diag["pen_max"] > 0).any():
            d64 = lambda t: type(t)(*[np.asarray(a, np.float64) if np.asarray(a).dtype != bool else a for a in t])
            o64_st, o64_sh, _ = o64.frame_step(d64(st), d64(sh), c(sp), c(spn), c(vw), st.dpdem_floe_eligible,
                                               c(vws))
            gst, gsh = to_gpu_state(st, sh, torch.float32)
            r_st, r_sh, r_diag = _frame(fs, gst, gsh, g, prefix, f, torch.float32)
            ice, ship = to_np_state(r_st, r_sh)
            w = assert_frame_matches(ice, ship, o_st, o_sh, st, sh, r_diag, o_diag, where=f"frame {f}",
                                     o_ice64=o64_st, o_ship64=o64_sh)
            for k, v in w.items():
                worst[k] = max(worst.get(k, 0.0), v)
            checked += 1
        st, sh = o_st, o_sh
    assert checked > 0
    print(prefix, "worst error / tolerance per field:", {k: f"{v:.2e}" for k, v in worst.items()})
    fs.close()


@pytest.mark.parametrize("dtype", ["f32", "f64"])
@pytest.mark.parametrize("prefix", ["small", "window"])
def test_contact_sets_match_oracle(prefix, dtype, golden32, golden64):
    """The ice-ice contact set of every substep (the pairs whose contact term
    the force phase computed) equals the oracle's all-pairs set (pairs with
    overlap > 0 and distance > 1e-6, jax_simulation.py:127-131), frame by
    frame from identical input states."""
    g = golden32 if dtype == "f32" else golden64
    npdt = np.float32 if dtype == "f32" else np.float64
    tdt = torch.float32 if dtype == "f32" else torch.float64
    fs = gpu_frame_step(g, prefix, tdt)
    rec = fs.record_contacts()
    o = make_oracle(g, prefix, npdt, pair_mode="all" if prefix == "small" else "grid")
    st, sh = initial_state(g, prefix, npdt)
    k = fs.n_ice_steps
    n_frames = min(g[f"{prefix}_pos"].shape[0], 150)
    total = 0
    for f in range(n_frames):
        sp, spn, vw, vws = frame_inputs(g, prefix, f)
        c = lambda a: np.asarray(a, np.float64).astype(npdt)
        o.contact_log = []
        o_st, o_sh, _ = o.frame_step(st, sh, c(sp), c(spn), c(vw), st.dpdem_floe_eligible, c(vws))
        gst, gsh = to_gpu_state(st, sh, tdt)
        _frame(fs, gst, gsh, g, prefix, f, tdt)
        sets, raw = rec.substeps(k)
        total += contact_sets_match(sets, raw, o.contact_log, o_st.elem_active, where=f"frame {f}")
        st, sh = o_st, o_sh
    assert total > 0, "the scenario must have ice-ice contacts"
    print(prefix, dtype, "contact pairs compared:", total)
    fs.close()


def test_scan_equals_frame_loop_and_phased_equals_persistent(golden32):
    from mbd_icenav_b200 import _abi
    g = golden32
    prefix = "window"
    fs = gpu_frame_step(g, prefix, torch.float32)
    o_st, o_sh = initial_state(g, prefix, np.float32)
    st0, sh0 = to_gpu_state(o_st, o_sh, torch.float32)
    K = 3
    d = torch.device("cuda", 0)
    rows = np.stack([np.concatenate(frame_inputs(g, prefix, f)[:2]) for f in range(K)])
    vw = np.stack([frame_inputs(g, prefix, f)[2] for f in range(K)])
    vws = np.stack([frame_inputs(g, prefix, f)[3] for f in range(K)])
    t = lambda a: torch.as_tensor(np.asarray(a, np.float64)).to(d, torch.float32)
    fin, fsh, hist = fs.scan_segment(st0, sh0, t(rows), t(vw), t(vws))
    st, sh = st0, sh0
    for f in range(K):
        st, sh, _ = _frame(fs, st, sh, g, prefix, f, torch.float32)
        assert torch.equal(hist[0][f], st.positions)
        assert torch.equal(hist[2][f], st.bond_intact)
        assert torch.equal(hist[3][f], sh.eta)
    for a, b in zip(fin, st):
        assert torch.equal(a, b)
    fs.set_launch_mode(_abi.DEM_LAUNCH_PHASED)
    fin2, fsh2, hist2 = fs.scan_segment(st0, sh0, t(rows), t(vw), t(vws))
    for a, b in zip(fin, fin2):
        assert torch.equal(a, b)
    for a, b in zip(hist, hist2):
        assert torch.equal(a, b)
    fs.close()


def test_f32_drift_1000_substeps_vs_f64_oracle(golden64):
    """Free-running fp32 GPU trajectory vs the fp64 oracle over 100 frames x 10 substeps."""
    g = golden64
    prefix = "small"
    fs = gpu_frame_step(g, prefix, torch.float32)
    o = make_oracle(g, prefix, np.float64, pair_mode="grid")
    o_st, o_sh = initial_state(g, prefix, np.float64)
    st, sh = to_gpu_state(o_st, o_sh, torch.float32)
    drift = []
    for f in range(100):
        sp, spn, vw, vws = frame_inputs(g, prefix, f)
        o_st, o_sh, _ = o.frame_step(o_st, o_sh, sp, spn, vw, o_st.dpdem_floe_eligible, vws)
        st, sh, _ = _frame(fs, st, sh, g, prefix, f, torch.float32)
        ice, ship = to_np_state(st, sh)
        drift.append(float(np.max(np.abs(ice.positions.astype(np.float64) - o_st.positions))))
    # fp32 positions near 200 m carry ~1e-5 m of rounding; the ship reaches the floes near
    # frame 80, so this window is dominated by rounding plus the first contacts
    assert max(drift) < 5e-3, drift
    print("max position drift (m) over 1000 substeps:", max(drift))
    fs.close()


def test_contact_in_hull_box_corner_is_not_culled():
    """A vertex inside the analytic hull's stern corner, farther from the ship
    centre than any outline point, still makes contact (pass 1 of
    jax_geometry.py:515-594); the reach bound must cover the hull box corners."""
    from mbd_icenav_b200 import sim
    from mbd_icenav_b200.config import SimulationConfig
    from mbd_icenav_b200.state import (build_static_arrays, initial_ice_state_arrays,
                                       ship_dynamics_arrays)
    from mbd_icenav_b200.vessel import ShipProperties, SupplyVessel, pointed_hull_outline
    from oracle.dem_oracle import OShip, OState, Oracle, params_from_config
    cfg = SimulationConfig()
    tri = np.array([[29.9, 5.9], [31.9, 6.2], [30.6, 7.9]])
    cent = tri.mean(axis=0, keepdims=True)
    props = ShipProperties(length=60.0, beam=12.0, draft=4.0)
    hull = pointed_hull_outline(60.0, 12.0)
    assert np.hypot(*tri[0]) > np.hypot(hull[:, 0], hull[:, 1]).max()
    sa = build_static_arrays([tri], cent, [], np.ones(1), None, cfg)
    sd = ship_dynamics_arrays(props, cfg, 60.0, 12.0, hull)
    sv = SupplyVessel(mass=props.mass, length=60.0)
    o = Oracle(sa, sd, params_from_config(cfg, 60.0, 12.0, 1, 0.05, 0.05, False, 1.0), sv.B)
    st0 = OState(*initial_ice_state_arrays(1, cent, 0, np.zeros(1, np.int32)))
    sh0 = OShip(np.zeros(3), np.zeros(3), np.zeros(6), np.zeros(3))
    _, _, od = o.frame_step(st0, sh0, np.zeros(3), np.zeros(3), np.zeros((1, 2)), st0.dpdem_floe_eligible)
    assert od["pen_max"][0] > 0
    fs = sim.make_frame_step(sa, cfg, sd, 60.0, 12.0, 1, 0.05, 0.05, False, sv.B, 1.0,
                             device=torch.device("cuda", 0), dtype=torch.float64)
    st, sh = to_gpu_state(st0, sh0, torch.float64)
    z = torch.zeros(3, dtype=torch.float64, device="cuda")
    _, _, diag = fs(st, sh, z, z, torch.zeros((1, 2), dtype=torch.float64, device="cuda"),
                    st.dpdem_floe_eligible)
    np.testing.assert_allclose(diag["pen_max"].cpu().numpy(), od["pen_max"], rtol=1e-12)
    fs.close()
