"""GPU parity: libdem_b200 (through its C ABI) vs the reference's outputs and the oracle.

* float64 free runs vs the golden vectors (the reference's own code);
* float32 single frames from identical input states vs the float32 oracle:
  positions/velocities within 1e-5 (norm-wise relative), contact set,
  bond-intact, activation and eligibility masks equal;
* scan == frame loop and persistent == phased launches, bit for bit;
* float32 drift over 1,000 substeps against the float64 oracle.
"""
import numpy as np
import pytest

from helpers import (frame_inputs, gpu_frame_step, initial_state, make_oracle, rel_err, to_gpu_state,
                     to_np_state)

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

F32_TOL = 1e-5  # per-step relative tolerance in fp32


def _frame(fs, st, sh, g, prefix, f, dtype):
    sp, spn, vw, vws = frame_inputs(g, prefix, f)
    d = torch.device("cuda", 0)
    t = lambda a: torch.as_tensor(np.asarray(a, np.float64)).to(d, dtype)
    return fs(st, sh, t(sp), t(spn), t(vw), st.dpdem_floe_eligible, t(vws))


@pytest.mark.parametrize("prefix", ["hex", "small", "window"])
def test_f64_free_run_matches_reference(prefix, golden64):
    g = golden64
    fs = gpu_frame_step(g, prefix, torch.float64)
    o_st, o_sh = initial_state(g, prefix, np.float64)
    st, sh = to_gpu_state(o_st, o_sh, torch.float64)
    n_frames = g[f"{prefix}_pos"].shape[0]
    worst = 0.0
    for f in range(n_frames):
        st, sh, diag = _frame(fs, st, sh, g, prefix, f, torch.float64)
        ice, ship = to_np_state(st, sh)
        e = max(rel_err(ice.positions, g[f"{prefix}_pos"][f], 1e-6),
                rel_err(ice.velocities, g[f"{prefix}_vel"][f], 1e-3),
                rel_err(ship.eta, g[f"{prefix}_eta"][f]))
        worst = max(worst, e)
        assert e < 1e-6, (f, e)
        np.testing.assert_array_equal(ice.bond_intact, g[f"{prefix}_intact"][f], err_msg=f"frame {f}")
        np.testing.assert_array_equal(ice.elem_active, g[f"{prefix}_active"][f])
        np.testing.assert_array_equal(ice.dpdem_floe_eligible, g[f"{prefix}_elig"][f])
        np.testing.assert_array_equal(diag["pen_max"].cpu().numpy() > 0, g[f"{prefix}_pen"][f] > 0)
        assert rel_err(diag["force_mag"].cpu().numpy(), g[f"{prefix}_fmag"][f], 1.0) < 1e-6
    fs.close()


@pytest.mark.parametrize("prefix", ["hex", "small", "window"])
def test_f32_single_frames_match_oracle(prefix, golden32):
    """Same fp32 input state -> one frame on GPU and in the fp32 oracle."""
    g = golden32
    fs = gpu_frame_step(g, prefix, torch.float32)
    o = make_oracle(g, prefix, np.float32, pair_mode="grid")
    st, sh = initial_state(g, prefix, np.float32)
    n_frames = g[f"{prefix}_pos"].shape[0]
    checked = 0
    for f in range(n_frames):
        sp, spn, vw, vws = frame_inputs(g, prefix, f)
        c = lambda a: np.asarray(a, np.float64).astype(np.float32)
        o_st, o_sh, o_diag = o.frame_step(st, sh, c(sp), c(spn), c(vw), st.dpdem_floe_eligible, c(vws))
        if prefix != "small" or f % 5 == 0 or (o_diag["pen_max"] > 0).any():
            gst, gsh = to_gpu_state(st, sh, torch.float32)
            r_st, r_sh, r_diag = _frame(fs, gst, gsh, g, prefix, f, torch.float32)
            ice, ship = to_np_state(r_st, r_sh)
            np.testing.assert_array_equal(r_diag["pen_max"].cpu().numpy() > 0, o_diag["pen_max"] > 0)
            assert rel_err(ice.positions, o_st.positions, 1e-6) < F32_TOL, f
            assert rel_err(ice.velocities, o_st.velocities, 1e-3) < F32_TOL * 10, f
            assert rel_err(ice.rotations, o_st.rotations, 1e-6) < F32_TOL, f
            assert rel_err(ice.submergence, o_st.submergence, 1e-6) < F32_TOL, f
            np.testing.assert_array_equal(ice.bond_intact, o_st.bond_intact, err_msg=f"frame {f}")
            np.testing.assert_array_equal(ice.elem_active, o_st.elem_active)
            np.testing.assert_array_equal(ice.dpdem_floe_eligible, o_st.dpdem_floe_eligible)
            assert rel_err(ship.eta, o_sh.eta) < F32_TOL
            checked += 1
        st, sh = o_st, o_sh
    assert checked > 0
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
