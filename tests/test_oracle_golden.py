"""Pin the oracle: NumPy restatement vs the reference's own code (golden vectors).

The golden files were produced by executing the reference's unmodified
``medea_ice_ship/jax_*.py`` on the NumPy ``jax`` shim
(``tests/golden/make_golden.py``).  float64 comparisons use a 1e-9 norm-wise
tolerance (identical formulas, identical operation order); float32 ones a
few ulps; every boolean (contact, intact, active, eligible) must be equal.
"""
import numpy as np
import pytest

from helpers import (B_THRUST, fn_static, frame_inputs, initial_state, make_oracle,
                     rel_err, scenario_params, shipdyn_from_golden, static_from_golden)
from oracle.dem_oracle import (OParams, OShip, OState, Oracle, bond_damage_update,
                               grid_pairs, params_from_config, ship_step)

TOL = {np.float64: 1e-9, np.float32: 2e-5}


def _fn_oracle(g, dtype):
    cfg_params = params_from_config(__import__("helpers").default_cfg(), 40.0, 8.0, 1, 0.05,
                                    0.005, False, 1.0)
    return Oracle(fn_static(g), shipdyn_from_golden(g, "fn"), cfg_params, B_THRUST, dtype=dtype)


def _fn_state(g, dtype):
    n = int(g["fn_npoly"])
    st = fn_static(g)
    nb = st.bond_i.shape[0]
    f = lambda k: np.asarray(g[k], np.float64).astype(dtype)
    return OState(positions=f("fn_pos"), velocities=f("fn_vel"), rotations=f("fn_rot"),
                  angular_vels=f("fn_avel"), submergence=f("fn_sub"),
                  bond_intact=np.asarray(g["fn_intact"], bool), bond_damage=f("fn_damage"),
                  bond_delta_m_0=np.zeros(nb, dtype), bond_delta_m_max=np.zeros(nb, dtype),
                  bond_delta_s=np.zeros(nb, dtype), elem_active=np.asarray(g["fn_active"], bool),
                  dpdem_floe_eligible=np.zeros(10, bool))


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_substep_functions(prec, golden64, golden32):
    g = golden64 if prec == "f64" else golden32
    dtype = np.float64 if prec == "f64" else np.float32
    o = _fn_oracle(g, dtype)
    st = _fn_state(g, dtype)
    fb, mb = o.bond_forces(st)
    fi, mi = o.ice_ice_forces(st)
    fd = o.drag(st, np.asarray(g["fn_vw"], np.float64).astype(dtype))
    md = o.rot_drag(st)
    tol = TOL[dtype]
    assert rel_err(fb, g["fn_bond_f"]) <= tol and rel_err(mb, g["fn_bond_m"]) <= tol
    assert rel_err(fi, g["fn_ice_f"]) <= tol and rel_err(mi, g["fn_ice_m"]) <= tol
    assert rel_err(fd, g["fn_drag"]) <= tol and rel_err(md, g["fn_rdrag"]) <= tol
    # integration with a dt_ice of 0.005 and the default clips
    o.p.dt_ice = 0.005
    it = o.integrate(st, np.asarray(g["fn_int_forces"], np.float64).astype(dtype),
                     np.asarray(g["fn_int_moments"], np.float64).astype(dtype))
    for a, k in ((it.positions, "fn_int_pos"), (it.velocities, "fn_int_vel"),
                 (it.rotations, "fn_int_rot"), (it.angular_vels, "fn_int_avel")):
        assert rel_err(a, g[k]) <= tol, k


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_restated_broad_phase_is_exact(prec, golden64, golden32):
    """Grid-candidate pairs give bitwise the same forces as all pairs."""
    g = golden64 if prec == "f64" else golden32
    dtype = np.float64 if prec == "f64" else np.float32
    o = _fn_oracle(g, dtype)
    st = _fn_state(g, dtype)
    f_all, m_all = o.ice_ice_forces(st)
    o.pair_mode = "grid"
    f_grid, m_grid = o.ice_ice_forces(st)
    np.testing.assert_array_equal(f_all, f_grid)
    np.testing.assert_array_equal(m_all, m_grid)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_ship_contact(prec, golden64, golden32):
    g = golden64 if prec == "f64" else golden32
    dtype = np.float64 if prec == "f64" else np.float32
    o = _fn_oracle(g, dtype)
    o.p.half_len, o.p.half_beam = 20.0, 4.0
    st = _fn_state(g, dtype)
    for k, (sx, sy, sp) in enumerate(np.asarray(g["fn_ship_poses"], np.float64)):
        pen, nx, ny = o.ship_contact(st.positions, st.rotations, dtype(sx), dtype(sy), dtype(sp))
        ref = g[f"fn_contact_{k}"]
        np.testing.assert_array_equal(pen > 0, ref[0] > 0)
        assert rel_err(pen, ref[0]) <= TOL[dtype]
        hit = ref[0] > 0
        assert rel_err(nx[hit], ref[1][hit], 1.0) <= TOL[dtype]
        assert rel_err(ny[hit], ref[2][hit], 1.0) <= TOL[dtype]


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_bond_damage_update(prec, golden64, golden32):
    g = golden64 if prec == "f64" else golden32
    dtype = np.float64 if prec == "f64" else np.float32
    dn, ds, sn, stt, sb, cd, cmax, c0 = [np.asarray(a, np.float64).astype(dtype) for a in g["fn_bd_in"]]
    intact = np.asarray(g["fn_bd_intact"], bool)
    d, mx, m0, it = bond_damage_update(dn, ds, sn, stt, sb, 1.8e6, 0.7, 12.0, 12.0, 1.75,
                                       cd, cmax, c0, intact, dtype)
    ref = g["fn_bd_out"]
    assert rel_err(d, ref[0]) <= TOL[dtype]
    assert rel_err(mx, ref[1]) <= TOL[dtype]
    assert rel_err(m0, ref[2]) <= TOL[dtype]
    np.testing.assert_array_equal(it, g["fn_bd_out_intact"])


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_ship_step(prec, golden64, golden32):
    g = golden64 if prec == "f64" else golden32
    dtype = np.float64 if prec == "f64" else np.float32
    sd = shipdyn_from_golden(g, "fn")
    f = lambda a: np.asarray(a, np.float64).astype(dtype)
    for row in np.asarray(g["fn_ship_rows"], np.float64):
        eta, nu, na, ei = row[0:3], row[3:6], row[6:12], row[12:15]
        sp, spn, tau, vws = row[15:18], row[18:21], row[21:24], row[24:26]
        auto = bool(row[26])
        out = row[27:]
        r = ship_step(f(eta), f(nu), f(na), f(ei), f(sp), f(spn), f(tau), f(sd.M3inv), f(sd.D3),
                      f(sd.Kp), f(sd.Kd), f(sd.Ki), f(sd.B_pinv), f(sd.n_max), f(B_THRUST), 1.0,
                      0.05, f(vws), auto, (15.0, 8.0, 0.15), dtype)
        got = np.concatenate([np.asarray(x, np.float64) for x in r])
        np.testing.assert_allclose(got, out, rtol=10 * TOL[dtype], atol=10 * TOL[dtype] * np.abs(out).max())


def test_known_answer_vessel_constants():
    """Fossen bis-scaled supply-vessel matrices (the reference tests' known answers)."""
    import math
    from mbd_icenav_b200.vessel import SupplyVessel
    v = SupplyVessel()
    L = 76.2
    T = np.diag([1.0, 1.0, L])
    Mb = np.array([[1.1274, 0, 0], [0, 1.8902, -0.0744], [0, -0.0744, 0.1278]])
    Db = np.array([[0.0358, 0, 0], [0, 0.1183, -0.0124], [0, -0.0041, 0.0308]])
    np.testing.assert_allclose(v.M3, 6000e3 * T @ Mb @ T, rtol=1e-10)
    np.testing.assert_allclose(v.D3, 6000e3 * math.sqrt(9.81 / L) * T @ Db @ T, rtol=1e-10)
    np.testing.assert_allclose(v.M3 @ v.M3inv, np.eye(3), atol=1e-8)
    np.testing.assert_allclose(v.B, B_THRUST, rtol=1e-10)
    assert v.T_n == 1.0
    np.testing.assert_array_equal(v.n_max, [250, 250, 250, 250, 160, 160])
    # max tunnel thrust 3.2 * 250^2 = 200 kN
    assert abs(v.B[1, 0] * 250.0 ** 2 - 200e3) < 1e-6


SEQ_FIELDS = (("pos", "positions"), ("vel", "velocities"), ("rot", "rotations"),
              ("avel", "angular_vels"), ("sub", "submergence"), ("damage", "bond_damage"))


def _run_sequence(g, prefix, dtype, n_frames, pair_mode="all"):
    o = make_oracle(g, prefix, dtype, pair_mode)
    st, ship = initial_state(g, prefix, dtype)
    outs = []
    for f in range(n_frames):
        sp, spn, vw, vws = frame_inputs(g, prefix, f)
        st, ship, diag = o.frame_step(st, ship, sp.astype(dtype), spn.astype(dtype),
                                      vw.astype(dtype), st.dpdem_floe_eligible, vws.astype(dtype))
        outs.append((st, ship, diag))
    return outs


@pytest.mark.parametrize("prefix,prec", [("hex", "f64"), ("hex", "f32"), ("small", "f64"),
                                         ("small", "f32"), ("window", "f64"), ("window", "f32")])
def test_frame_sequence(prefix, prec, golden64, golden32):
    g = golden64 if prec == "f64" else golden32
    dtype = np.float64 if prec == "f64" else np.float32
    n_frames = g[f"{prefix}_pos"].shape[0]
    outs = _run_sequence(g, prefix, dtype, n_frames, pair_mode="grid" if prefix != "hex" else "all")
    tol = TOL[dtype]
    for f, (st, ship, diag) in enumerate(outs):
        for gk, sk in SEQ_FIELDS:
            assert rel_err(getattr(st, sk), g[f"{prefix}_{gk}"][f], 1e-6) <= tol, (f, gk)
        np.testing.assert_array_equal(st.bond_intact, g[f"{prefix}_intact"][f], err_msg=f"intact {f}")
        np.testing.assert_array_equal(st.elem_active, g[f"{prefix}_active"][f])
        np.testing.assert_array_equal(st.dpdem_floe_eligible, g[f"{prefix}_elig"][f])
        np.testing.assert_array_equal(diag["pen_max"] > 0, g[f"{prefix}_pen"][f] > 0)
        assert rel_err(diag["pen_max"], g[f"{prefix}_pen"][f], 1e-6) <= tol
        assert rel_err(diag["force_mag"], g[f"{prefix}_fmag"][f], 1.0) <= tol
        assert rel_err(ship.eta, g[f"{prefix}_eta"][f]) <= tol
        assert rel_err(ship.nu, g[f"{prefix}_nu"][f], 1e-3) <= tol
        assert rel_err(diag["F_ice_on_ship"], g[f"{prefix}_F"][f], 1.0) <= tol
        assert rel_err(diag["J_cumul_incr"], g[f"{prefix}_J"][f], 1e-3) <= tol


def test_scan_matches_frame_loop(golden64):
    """Chunked scan == per-frame loop (``test_jax_full_scan.py:233-295`` analogue)."""
    g = golden64
    o = make_oracle(g, "small", np.float64, "grid")
    st, ship = initial_state(g, "small", np.float64)
    sp = np.asarray(g["small_setpoints"], np.float64)[:50]
    n = st.positions.shape[0]
    _, _, hist = o.scan_segment(st, ship, sp, np.zeros((50, n, 2)), np.zeros((50, 2)))
    np.testing.assert_allclose(hist["positions"], g["small_scan50_pos"], rtol=1e-8, atol=1e-8)
    np.testing.assert_allclose(hist["eta"], g["small_scan50_eta"], rtol=1e-8, atol=1e-8)
    np.testing.assert_allclose(hist["positions"], g["small_pos"][:50], rtol=1e-8, atol=1e-8)


def test_grid_pairs_exact_set():
    rng = np.random.default_rng(0)
    pos = rng.uniform(0, 50, (400, 2))
    r = rng.uniform(0.5, 2.0, 400)
    pi, pj = grid_pairs(pos, r)
    d = np.linalg.norm(pos[:, None] - pos[None], axis=-1)
    ii, jj = np.nonzero(np.triu(d < r[:, None] + r[None, :], 1))
    got = set(zip(pi.tolist(), pj.tolist()))
    want = set(zip(ii.tolist(), jj.tolist()))
    assert want <= got
    assert np.all(np.diff(pi * 1000 + pj) > 0)
