"""Host side of the batched planner rollouts (no GPU).

Window cutting, the batched static data of uneven windows (bonds and floes
renumbered per window, nothing crossing a window), control sampling and the
ice-free path model that places the windows.
"""
import numpy as np

from mbd_icenav_b200 import rollouts, scene
from mbd_icenav_b200.config import DEFAULT_MATERIAL, get_default_simulation_config
from mbd_icenav_b200.state import build_static_arrays, ship_dynamics_arrays


def _field():
    return scene.make_small_field(seed=3, n_frames=4)


def test_sample_controls_are_clipped_gaussians_without_sway():
    rng = np.random.default_rng(0)
    u = rollouts.sample_controls(rng, 512, 64, nominal=(5e4, 0.0))
    assert u.shape == (64, 512, 3)
    assert np.all(u[..., 1] == 0.0)
    assert np.all(np.abs(u[..., 0]) <= rollouts.SURGE_MAX)
    assert np.all(np.abs(u[..., 2]) <= rollouts.YAW_MAX)
    # sigma = 0.3 of the maximum, around the nominal (few samples reach the clip)
    assert abs(u[..., 0].mean() - 5e4) < 0.02 * rollouts.SURGE_MAX
    assert abs(u[..., 0].std() / rollouts.SURGE_MAX - 0.3) < 0.02
    assert abs(u[..., 2].std() / rollouts.YAW_MAX - 0.3) < 0.02


def test_predicted_paths_follow_the_vessel_model():
    f = _field()
    sd = ship_dynamics_arrays(f.ship_props, get_default_simulation_config(), f.ship_length, f.ship_beam,
                              f.hull_local)
    eta0 = np.array([10.0, 20.0, 0.3])
    # at rest with no control the ship stays where it is
    still = rollouts.predict_paths(eta0, np.zeros(3), np.zeros((5, 2, 3)), sd.M3inv, sd.D3, 0.05)
    np.testing.assert_array_equal(still, np.broadcast_to(eta0, still.shape))
    # the surge force that holds 2 m/s against linear damping keeps 2 m/s along the heading
    nu0 = np.array([2.0, 0.0, 0.0])
    u = np.zeros((40, 1, 3))
    u[..., 0] = (np.asarray(sd.D3) @ nu0)[0]
    path = rollouts.predict_paths(eta0, nu0, u, sd.M3inv, sd.D3, 0.05)
    step = np.diff(path[:, 0, :2], axis=0)
    np.testing.assert_allclose(np.linalg.norm(step, axis=1), 2.0 * 0.05, rtol=1e-9)
    np.testing.assert_allclose(np.arctan2(step[:, 1], step[:, 0]), 0.3, atol=1e-9)


def test_windows_are_the_elements_nearest_each_path():
    f = _field()
    rng = np.random.default_rng(1)
    paths = np.stack([np.tile(f.centroids[rng.integers(f.n)], (3, 1)) for _ in range(4)], 1)  # (3, 4, 2)
    paths = np.concatenate([paths, np.zeros((3, 4, 1))], -1)
    sizes = [3, 7, 12, 20]
    wins = rollouts.cut_windows(f.centroids, paths, sizes)
    for q, w in enumerate(wins):
        assert len(w) == sizes[q] and np.all(np.diff(w) > 0)
        d = np.linalg.norm(f.centroids - paths[0, q, :2], axis=1)
        inside, outside = d[w], np.delete(d, w)
        assert inside.max() <= outside.min() + 1e-12


def test_batched_static_of_overlapping_uneven_windows():
    f = _field()
    cfg = get_default_simulation_config()
    st = build_static_arrays(f.polygons, f.centroids, f.bonds, f.thicknesses, f.parent_ids, cfg, DEFAULT_MATERIAL,
                             0.05)
    wins = [np.arange(0, 10), np.arange(5, 24), np.array([2, 3, 4, 17])]  # overlapping, uneven
    bs, ss = rollouts.window_static(st, wins)
    np.testing.assert_array_equal(ss, [0, 10, 29, 33])
    assert bs.masses.shape == (33,)
    np.testing.assert_array_equal(bs.masses, np.concatenate([st.masses[w] for w in wins]))
    sys_of = np.repeat(np.arange(3), np.diff(ss))
    # every bond lies inside one window and is a bond of the field between the same elements
    assert np.all(sys_of[bs.bond_i] == sys_of[bs.bond_j])
    orig = {(min(i, j), max(i, j)) for i, j in zip(st.bond_i.tolist(), st.bond_j.tolist())}
    allw = np.concatenate(wins)
    for i, j in zip(bs.bond_i.tolist(), bs.bond_j.tolist()):
        a, b = int(allw[i]), int(allw[j])
        assert (min(a, b), max(a, b)) in orig
    # and every field bond with both ends in a window appears in that window
    for q, w in enumerate(wins):
        inside = set(w.tolist())
        want = sum(1 for i, j in orig if i in inside and j in inside)
        assert int(np.sum(sys_of[bs.bond_i] == q)) == want
    # floes are renumbered densely and never span two windows
    floe = bs.initial_floe_of
    assert floe.min() == 0 and len(np.unique(floe)) == floe.max() + 1
    for fl in np.unique(floe):
        assert len(np.unique(sys_of[floe == fl])) == 1


def test_ice_edge_pose_puts_the_bow_short_of_the_first_floe():
    f = _field()
    pose = rollouts.ice_edge_pose(f, gap=3.0)
    d = np.array([np.cos(pose[2]), np.sin(pose[2])])
    rel = f.centroids - pose[:2]
    along = rel @ d
    across = np.abs(rel @ np.array([-d[1], d[0]]))
    ahead = along[(along > 0) & (across < 0.5 * f.ship_beam)]
    np.testing.assert_allclose(ahead.min(), 0.5 * f.ship_length + 3.0, rtol=1e-12)
    assert pose[2] == f.trajectory[0][2]
