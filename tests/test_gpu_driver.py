"""The chunked driver (simulate_jax_chunked_replan) on the GPU.

Path equivalence as the reference's tests check it (test_jax_chunked_replan.py:
68-160: chunked vs full scan vs per-frame): the histories of a run in chunks
of 25 frames (the last one padded) equal those of a single 70-frame chunk and
those of a plain frame-by-frame loop, bit for bit; goal-line trimming keeps
the frames up to and including the first crossing; histories stay on the
device until read.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

N_FRAMES = 70


@pytest.fixture(scope="module")
def field():
    from mbd_icenav_b200 import scene
    f = scene.make_small_field(seed=0, n_frames=N_FRAMES)
    f.trajectory = f.trajectory + np.array([0.0, 27.0, 0.0])  # meet the floes within the run
    return f


def _run(f, chunk, **kw):
    from mbd_icenav_b200 import driver
    return driver.simulate_jax_chunked_replan(
        f.polygons, f.centroids, f.bonds, f.trajectory[0, :2], f.ship_length, f.ship_beam, N_FRAMES, f.dt,
        (0.0, 0.0), f.thicknesses, f.ship_props, ship_trajectory=f.trajectory, replan_every_n_frames=chunk,
        parent_ids=f.parent_ids, verbose=False, n_ice_steps=f.n_ice_steps, hull_local=f.hull_local,
        dilation=0.05, dtype=torch.float64, device="cuda", **kw)


def test_chunked_equals_single_chunk_and_frame_loop(field):
    f = field
    a = _run(f, 25, return_ship_diagnostics=True)
    b = _run(f, None, return_ship_diagnostics=True)
    for i in (0, 1, 2, 4):
        assert len(a[i]) == len(b[i]) == N_FRAMES + 1
        np.testing.assert_array_equal(a[i].to_numpy(), b[i].to_numpy())
    assert len(a[3]) == N_FRAMES
    for (pa, ha), (pb, hb) in zip(a[3], b[3]):
        np.testing.assert_array_equal(pa, pb)
        assert ha == hb
    assert a[5][-1]["impulse_cumul"] == b[5][-1]["impulse_cumul"]
    assert a[5][-1]["impulse_cumul"] > 0.0  # the ship met the ice
    # a plain frame loop through the same kind of context
    from mbd_icenav_b200.sim import build_sim_context
    from mbd_icenav_b200.state import build_initial_ice_state, build_initial_ship_state
    ctx = build_sim_context(f.polygons, f.centroids, f.bonds, f.trajectory[0, :2], f.ship_length, f.ship_beam,
                            N_FRAMES, f.dt, (0.0, 0.0), f.thicknesses, f.ship_props, parent_ids=f.parent_ids,
                            verbose=False, n_ice_steps=f.n_ice_steps, hull_local=f.hull_local, dilation=0.05,
                            dtype=torch.float64, device="cuda")
    fs = ctx.frame_step
    st = build_initial_ice_state(len(f.polygons), f.centroids, len(f.bonds),
                                 ctx.static.initial_floe_of.cpu().numpy(), dtype=torch.float64, device="cuda")
    sh = build_initial_ship_state(f.trajectory[0, :2], float(f.trajectory[0, 2]), dtype=torch.float64,
                                  device="cuda")
    d = torch.device("cuda", 0)
    zw = torch.zeros((len(f.polygons), 2), dtype=torch.float64, device=d)
    z2 = torch.zeros(2, dtype=torch.float64, device=d)
    for fr in range(N_FRAMES):
        sp = torch.as_tensor(f.trajectory[fr], dtype=torch.float64, device=d)
        spn = torch.as_tensor(f.trajectory[fr + 1], dtype=torch.float64, device=d)
        st, sh, _ = fs(st, sh, sp, spn, zw, st.dpdem_floe_eligible, z2)
        np.testing.assert_array_equal(st.positions.cpu().numpy(), a[0][fr + 1], err_msg=f"frame {fr}")
        np.testing.assert_array_equal(st.bond_intact.cpu().numpy(), a[2][fr + 1])


def test_goal_line_trims_at_the_first_crossing(field):
    f = field
    full = _run(f, 25)
    ys = np.array([p[1] for p, _ in full[3]])
    tol = 15.0
    goal = float(ys[40]) + tol  # first crossed at frame 40 (the ship moves north monotonically)
    first = int(np.argmax(ys >= goal - tol))
    out = _run(f, 25, goal_y_line=goal, goal_tolerance=tol)
    assert len(out[3]) == first + 1
    assert len(out[0]) == first + 2
    np.testing.assert_array_equal(out[0].to_numpy(), full[0].to_numpy()[:first + 2])


def test_histories_stay_on_the_device_until_read(field):
    out = _run(field, 25)
    pos = out[0]
    assert pos.tensor.is_cuda
    assert isinstance(pos[3], np.ndarray) and pos[3].shape == (len(field.polygons), 2)
    assert len(pos[2:5]) == 3
    with pytest.raises(IndexError):
        pos[len(pos)]
