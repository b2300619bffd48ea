"""Planner rollouts: the frame step with each ship driven by controls.

CPU: the oracle's control-driven vessel step equals the reference's own
``ship_euler_step_jax`` + ``_clip_velocity_jax`` composition bit for bit
(``tests/golden/rollout_golden.npz``).

GPU: two window systems with different random controls, stepped together by
``dem_rollout_segment``, follow the oracle's frame loop with the same controls
(float64, within 1e-9; bond, activation and eligibility masks equal).
"""
import os

import numpy as np
import pytest

from oracle.dem_oracle import ship_step

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "rollout_golden.npz")


def test_oracle_control_step_matches_reference():
    g = np.load(GOLDEN)
    z = np.zeros(3)
    for i in range(len(g["eta"])):
        e, nu, na, ei = ship_step(g["eta"][i], g["nu"][i], np.ones(6), np.full(3, 2.0), z, z, g["tau_ice"][i],
                                  g["M3inv"], g["D3"], None, None, None, None, None, None, 1.0, float(g["dt"]),
                                  g["vws"][i], False, g["vc"], np.float64, u_ctrl=g["u"][i])
        np.testing.assert_array_equal(e, g["eta_out"][i])
        np.testing.assert_array_equal(nu, g["nu_out"][i])
        np.testing.assert_array_equal(na, np.ones(6))       # RPMs kept
        np.testing.assert_array_equal(ei, np.full(3, 2.0))  # integral error kept


@pytest.mark.gpu
def test_gpu_rollouts_follow_the_oracle(golden64):
    torch = pytest.importorskip("torch")
    from test_gpu_batched import _batched_static
    from helpers import (B_THRUST, SCENARIOS, default_cfg, frame_inputs, initial_state, make_oracle, rel_err,
                         shipdyn_from_golden, static_from_golden, to_gpu_state, to_np_state)
    from mbd_icenav_b200 import sim
    from mbd_icenav_b200.config import IceMaterial
    g = golden64
    prefix = "window"
    Q, K = 2, 3
    L, B, k, dt_f, dti, auto, flex = SCENARIOS[prefix]
    st1 = static_from_golden(g, prefix)
    stq, n = _batched_static(st1, Q)
    fs = sim.make_frame_step(stq, default_cfg(), shipdyn_from_golden(g, prefix), L, B, k, dt_f, dti, auto,
                             B_THRUST, 1.0, material=IceMaterial(flexural_strength_base=flex),
                             device=torch.device("cuda", 0), dtype=torch.float64, system_start=[0, n, 2 * n])
    rng = np.random.default_rng(3)
    u = np.stack([rng.normal(0, 6e5, (K, Q)), np.zeros((K, Q)), rng.normal(0, 1.5e8, (K, Q))], -1)  # (K, Q, 3)
    o_st, o_sh = initial_state(g, prefix, np.float64)
    tile = lambda a: np.concatenate([np.asarray(a)] * Q, 0)
    bst = o_st._replace(**{f: tile(getattr(o_st, f)) for f in o_st._fields})
    bsh = o_sh._replace(**{f: np.tile(getattr(o_sh, f), (Q, 1)) for f in o_sh._fields})
    st, sh = to_gpu_state(bst, bsh, torch.float64)
    d = torch.device("cuda", 0)
    t = lambda a: torch.as_tensor(np.asarray(a, np.float64)).to(d, torch.float64)
    vw = np.stack([frame_inputs(g, prefix, f)[2] for f in range(K)])
    vws = np.stack([frame_inputs(g, prefix, f)[3] for f in range(K)])
    fin, fship, hist = fs.rollout_segment(st, sh, t(u), t(np.concatenate([vw] * Q, 1)),
                                          t(np.repeat(vws[:, None], Q, 1)))
    ice, ship = to_np_state(fin, fship)
    nb = int(np.asarray(st1.bond_i).shape[0])
    o = make_oracle(g, prefix, np.float64, pair_mode="grid")
    for q in range(Q):
        ost, osh = o_st, o_sh
        for f in range(K):
            ost, osh, _ = o.frame_step(ost, osh, np.zeros(3), np.zeros(3), vw[f], ost.dpdem_floe_eligible, vws[f],
                                       u_ctrl=u[f, q])
            np.testing.assert_allclose(hist[3][f, q].cpu().numpy(), osh.eta, rtol=1e-9, atol=1e-9)
        el, bo = slice(q * n, (q + 1) * n), slice(q * nb, (q + 1) * nb)
        assert rel_err(ice.positions[el], ost.positions, 1e-6) < 1e-9
        assert rel_err(ice.velocities[el], ost.velocities, 1e-3) < 1e-9
        np.testing.assert_array_equal(ice.bond_intact[bo], ost.bond_intact)
        np.testing.assert_array_equal(ice.elem_active[el], ost.elem_active)
        assert rel_err(ship.eta[q], osh.eta) < 1e-9
        assert rel_err(ship.nu[q], osh.nu, 1e-6) < 1e-9
    fs.close()


@pytest.mark.gpu
def test_gpu_uneven_windows_match_single_runs_and_costs():
    """Candidates on uneven windows cut from the medium field, started at the ice
    edge: the batched launch reproduces each candidate run alone bit for bit,
    and the device costs match the oracle's on the same paths."""
    torch = pytest.importorskip("torch")
    from oracle.rollout_oracle import raw_components, transferred_ke
    from mbd_icenav_b200 import rollouts, scene
    from mbd_icenav_b200.config import DEFAULT_MATERIAL, get_default_simulation_config
    from mbd_icenav_b200.costmap import build_costmap_jax
    from mbd_icenav_b200.state import build_static_arrays, ship_dynamics_arrays, to_device
    from mbd_icenav_b200.vessel import SupplyVessel
    f = scene.make_medium_field(seed=1, n_frames=8)
    cfg = get_default_simulation_config()
    st = build_static_arrays(f.polygons, f.centroids, f.bonds, f.thicknesses, f.parent_ids, cfg, DEFAULT_MATERIAL,
                             0.05)
    sd = ship_dynamics_arrays(f.ship_props, cfg, f.ship_length, f.ship_beam, f.hull_local)
    sv = SupplyVessel(mass=f.ship_props.mass, length=f.ship_length)
    d, dt = torch.device("cuda", 0), torch.float64
    sdd = to_device(sd, dt, d)
    eta0 = rollouts.ice_edge_pose(f, gap=-0.5)  # bow already at the first floe
    nu0 = np.array([2.0, 0.0, 0.0])
    Q, H = 4, 8
    rng = np.random.default_rng(2)
    u = rollouts.sample_controls(rng, Q, H, nominal=(float((np.asarray(sd.D3) @ nu0)[0]), 0.0))
    paths = rollouts.predict_paths(eta0, nu0, u, sd.M3inv, sd.D3, f.dt)
    wins = rollouts.cut_windows(f.centroids, paths, [200, 350, 520, 700])
    mk = lambda w: rollouts.make_batch(st, sdd, cfg, f.ship_length, f.ship_beam, f.n_ice_steps, f.dt, sv.B, sv.T_n,
                                       f.centroids, w, eta0, nu0, dtype=dt, device=d)
    batch = mk(wins)
    assert list(np.diff(batch.system_start)) == [200, 350, 520, 700]
    res = rollouts.run(batch, u)
    ss = batch.system_start
    touched = 0
    for q in range(Q):
        one = mk([wins[q]])
        r1 = rollouts.run(one, u[:, q:q + 1])
        el = slice(int(ss[q]), int(ss[q + 1]))
        assert torch.equal(res.state.positions[el], r1.state.positions), q
        assert torch.equal(res.state.velocities[el], r1.state.velocities), q
        assert torch.equal(res.state.elem_active[el], r1.state.elem_active), q
        assert torch.equal(res.history[3][:, q], r1.history[3].reshape(H, 3)), q
        touched += int(r1.state.elem_active.any())
        one.frame_step.close()
    assert touched > 0  # some candidate met the ice
    half = 128.0 - 20.0
    cm, _ = build_costmap_jax(f.centroids, f.thicknesses, st.radii, eta0[0] - half, eta0[0] + half, eta0[1] - half,
                              eta0[1] + half, ship_length=f.ship_length, ship_beam=f.ship_beam, masses=st.masses,
                              device=d)
    goal = eta0[:2] + np.array([0.0, 200.0])
    out = rollouts.costs(batch, res, cm, goal, f.ship_length, f.ship_beam).cpu().numpy()
    poses = np.concatenate([batch.ship.eta.cpu().numpy()[None], res.history[3].cpu().numpy()], 0)  # (H+1, Q, 3)
    c32 = np.float32(rollouts.ACTION_CENTER)
    s32 = np.float32(rollouts.ACTION_SCALE)
    meta = dict(x_origin=cm.x_origin, y_origin=cm.y_origin, resolution=cm.resolution, rows=cm.rows, cols=cm.cols)
    for q in range(Q):
        un = (u[:, q].astype(np.float32) - c32) / s32
        ref = raw_components(poses[:, q], un, cm.cost_map, meta, goal, f.ship_length, f.ship_beam)
        np.testing.assert_allclose(out[q, :4], ref, rtol=1e-5, atol=1e-6, err_msg=f"candidate {q}")
    ke = transferred_ke(batch.frame_step._keep["masses"].cpu().numpy(), batch.state.velocities.cpu().numpy(),
                        res.state.velocities.cpu().numpy(), ss)
    np.testing.assert_allclose(out[:, 4], ke, rtol=1e-9, atol=1e-6)
    assert (out[:, 4] > 0).any()
    batch.frame_step.close()
