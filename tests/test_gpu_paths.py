"""GPU path equivalence and recovery, through the C ABI.

* A 100-frame scan equals the same frames run as three chunked scans, bit for
  bit, and follows the reference's own trajectory (the path-equivalence checks
  of the reference's tests, test_jax_full_scan.py:233-295 and
  test_jax_chunked_replan.py:68-160, which compare per-frame, full-scan and
  chunked runs).
* A handle created with neighbour-list and grid-bucket capacities far too
  small reports DEM_ERR_CAPACITY; the wrapper grows what overflowed and re-runs
  the call, and the result equals that of a handle sized right from the start.
"""
import numpy as np
import pytest

from helpers import frame_inputs, gpu_frame_step, initial_state, rel_err, to_gpu_state

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _scan_inputs(g, prefix, f0, f1, dtype):
    d = torch.device("cuda", 0)
    t = lambda a: torch.as_tensor(np.asarray(a, np.float64)).to(d, dtype)
    rows = np.stack([np.concatenate(frame_inputs(g, prefix, f)[:2]) for f in range(f0, f1)])
    vw = np.stack([frame_inputs(g, prefix, f)[2] for f in range(f0, f1)])
    vws = np.stack([frame_inputs(g, prefix, f)[3] for f in range(f0, f1)])
    return t(rows), t(vw), t(vws)


def test_chunked_scans_equal_one_scan_and_follow_the_reference(golden64):
    g = golden64
    prefix = "small"
    fs = gpu_frame_step(g, prefix, torch.float64)
    o_st, o_sh = initial_state(g, prefix, np.float64)
    st0, sh0 = to_gpu_state(o_st, o_sh, torch.float64)
    K = 100  # the ship meets the floes near frame 80
    full_st, full_sh, full_h = fs.scan_segment(st0, sh0, *_scan_inputs(g, prefix, 0, K, torch.float64))
    st, sh, hists = st0, sh0, []
    for f0, f1 in ((0, 40), (40, 75), (75, K)):
        st, sh, h = fs.scan_segment(st, sh, *_scan_inputs(g, prefix, f0, f1, torch.float64))
        hists.append(h)
    for a, b in zip(full_st, st):
        assert torch.equal(a, b)
    for a, b in zip(full_sh, sh):
        assert torch.equal(a, b)
    for i, full in enumerate(full_h):
        assert torch.equal(full, torch.cat([h[i] for h in hists]))
    pos = full_h[0].cpu().numpy()
    assert rel_err(pos, g[f"{prefix}_pos"][:K], 1e-6) < 1e-6
    np.testing.assert_array_equal(full_h[2].cpu().numpy(), g[f"{prefix}_intact"][:K])
    fs.close()


def test_capacity_overflow_is_retried_with_identical_results(golden32):
    g = golden32
    prefix = "window"
    o_st, o_sh = initial_state(g, prefix, np.float32)
    inputs = _scan_inputs(g, prefix, 0, 3, torch.float32)
    ref = gpu_frame_step(g, prefix, torch.float32)
    st, sh = to_gpu_state(o_st, o_sh, torch.float32)
    r_st, r_sh, r_h = ref.scan_segment(st, sh, *inputs)
    tight = gpu_frame_step(g, prefix, torch.float32, max_neighbors=6, bucket_capacity=6)
    st, sh = to_gpu_state(o_st, o_sh, torch.float32)
    t_st, t_sh, t_h = tight.scan_segment(st, sh, *inputs)
    info = tight.info()
    assert info["capacity_flags"] != 0  # something overflowed and was grown
    assert tight.params.max_neighbors > 6 or tight.params.bucket_capacity > 6
    for a, b in zip(r_st + r_sh, t_st + t_sh):
        assert torch.equal(a, b)
    for a, b in zip(r_h, t_h):
        assert torch.equal(a, b)
    ref.close()
    tight.close()


def test_results_do_not_depend_on_the_skin_or_the_escape_period(golden64):
    """Verlet lists are supersets of the touching pairs whatever the skin, and a
    skin wide enough for the largest move of one substep processes escapes only
    every second substep: the trajectories stay the same bit for bit."""
    from helpers import SCENARIOS, default_cfg
    g = golden64
    prefix = "small"
    K = 100
    _, _, _, _, dti, _, _ = SCENARIOS[prefix]
    vclip = float(default_cfg().velocity_clip[1])
    dmax = np.sqrt(2.0) * vclip * dti
    o_st, o_sh = initial_state(g, prefix, np.float64)
    runs = {}
    for skin in (0.3, 0.6, 1.2):
        fs = gpu_frame_step(g, prefix, torch.float64, skin=skin)
        st0, sh0 = to_gpu_state(o_st, o_sh, torch.float64)
        runs[skin] = (fs.scan_segment(st0, sh0, *_scan_inputs(g, prefix, 0, K, torch.float64)),
                      fs.info()["neighbor_rebuilds"])
        fs.close()
    assert 0.99 * (0.5 * 0.3 - dmax) < 0.25 * 0.3       # skin 0.3: every substep
    assert 0.99 * (0.5 * 0.6 - dmax) >= 0.25 * 0.6      # skin 0.6: every second substep
    (ref_st, ref_sh, ref_h), rounds_03 = runs[0.3]
    for skin in (0.6, 1.2):
        (st, sh, h), rounds = runs[skin]
        for a, b in zip(ref_st, st):
            assert torch.equal(a, b), skin
        for a, b in zip(ref_sh, sh):
            assert torch.equal(a, b), skin
        for a, b in zip(ref_h, h):
            assert torch.equal(a, b), skin
        assert rounds < rounds_03, skin  # fewer rebuild rounds
    assert rounds_03 > 0


def _split_runs(fs, st0, sh0, inputs):
    from mbd_icenav_b200 import _abi
    out = []
    for force_split, mark_split in ((_abi.DEM_SPLIT_AUTO, _abi.DEM_SPLIT_AUTO),
                                    (_abi.DEM_SPLIT_THREAD, _abi.DEM_SPLIT_WARP),
                                    (_abi.DEM_SPLIT_WARP, _abi.DEM_SPLIT_CTA)):
        fs.set_work_split(force_split, mark_split)
        out.append(fs.scan_segment(st0, sh0, *inputs))
    fs.set_work_split()
    return out


def _assert_same(runs):
    (st_a, sh_a, h_a) = runs[0]
    for st, sh, h in runs[1:]:
        for a, b in zip(st_a, st):
            assert torch.equal(a, b)
        for a, b in zip(sh_a, sh):
            assert torch.equal(a, b)
        for a, b in zip(h_a, h):
            assert torch.equal(a, b)


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_work_splits_give_identical_results_golden_field(golden64, dtype):
    """A thread or a warp per active element, a CTA or a warp per escaped element:
    the same trajectories bit for bit (the small scenario, through first contact)."""
    g = golden64
    dt = torch.float64 if dtype == "f64" else torch.float32
    fs = gpu_frame_step(g, "small", dt)
    o_st, o_sh = initial_state(g, "small", np.float64)
    st0, sh0 = to_gpu_state(o_st, o_sh, dt)
    runs = _split_runs(fs, st0, sh0, _scan_inputs(g, "small", 0, 100, dt))
    _assert_same(runs)
    assert runs[0][0].elem_active.any()  # the ship met the ice
    fs.close()


def test_work_splits_give_identical_results_ship_in_the_medium_field():
    """The same on the 12k-element medium field with the ship pushing into the ice
    edge for 40 frames (the forced splits run both paths on its active floes)."""
    from mbd_icenav_b200 import rollouts, scene
    from mbd_icenav_b200.sim import build_sim_context
    from mbd_icenav_b200.state import build_initial_ice_state, build_initial_ship_state
    f = scene.make_medium_field(seed=2, n_frames=40)
    K = 40
    eta0 = rollouts.ice_edge_pose(f, gap=0.5)
    d = np.array([np.cos(eta0[2]), np.sin(eta0[2])])
    path = np.array([[eta0[0] + 2.0 * 0.05 * i * d[0], eta0[1] + 2.0 * 0.05 * i * d[1], eta0[2]]
                     for i in range(K + 2)])
    ctx = build_sim_context(f.polygons, f.centroids, f.bonds, eta0[:2], f.ship_length, f.ship_beam, K, f.dt,
                            (0.0, 0.0), f.thicknesses, f.ship_props, parent_ids=f.parent_ids, verbose=False,
                            n_ice_steps=f.n_ice_steps, hull_local=f.hull_local, dilation=0.05,
                            dtype=torch.float32, device="cuda")
    fs = ctx.frame_step
    st0 = build_initial_ice_state(f.n, f.centroids, len(f.bonds), ctx.static.initial_floe_of.cpu().numpy(),
                                  dtype=torch.float32, device="cuda")
    sh0 = build_initial_ship_state(eta0[:2], float(eta0[2]), dtype=torch.float32, device="cuda")
    dev = torch.device("cuda", 0)
    rows = torch.as_tensor(np.concatenate([path[:K], path[1:K + 1]], 1), dtype=torch.float32, device=dev)
    vw = torch.zeros((K, f.n, 2), dtype=torch.float32, device=dev)
    runs = _split_runs(fs, st0, sh0, (rows, vw))
    _assert_same(runs)
    assert int(runs[0][0].elem_active.sum()) > 0  # the ship met the ice
    assert fs.info()["escaped_total"] > 0
    fs.close()


@pytest.mark.parametrize("k", [3, 4])
def test_lazy_escapes_with_odd_and_even_substep_counts(golden64, k):
    """Lazy escapes are taken at even substeps that have a successor in the frame;
    with 3 or 4 substeps per frame the trajectory at skin 2.4 m (lazy: wide enough
    for the longer substeps' largest move) equals the one at 0.3 m (every escape
    processed at once) bit for bit."""
    from mbd_icenav_b200 import sim
    from mbd_icenav_b200.config import IceMaterial
    from helpers import B_THRUST, SCENARIOS, default_cfg, shipdyn_from_golden, static_from_golden
    g = golden64
    L, B, _, dt, _, auto, flex = SCENARIOS["small"]
    o_st, o_sh = initial_state(g, "small", np.float64)
    dmax = np.sqrt(2.0) * float(default_cfg().velocity_clip[1]) * dt / k
    assert 0.99 * (0.5 * 2.4 - dmax) >= 0.25 * 2.4  # lazy mode at 2.4 m
    out = []
    for skin in (0.3, 2.4):
        fs = sim.make_frame_step(static_from_golden(g, "small"), default_cfg(), shipdyn_from_golden(g, "small"), L, B,
                                 k, dt, dt / k, auto, B_THRUST, 1.0, material=IceMaterial(flexural_strength_base=flex),
                                 device=torch.device("cuda", 0), dtype=torch.float64, skin=skin)
        st0, sh0 = to_gpu_state(o_st, o_sh, torch.float64)
        out.append(fs.scan_segment(st0, sh0, *_scan_inputs(g, "small", 0, 100, torch.float64)))
        fs.close()
    _assert_same(out)
    assert out[0][0].elem_active.any()


def test_medium_field_scan_equals_single_frame_calls():
    """A 40-frame call on the 12k-element medium field (its later frames skip
    the force chunks that stay frozen, far from the hull and dry in the cull
    and contact-force sweeps) equals 40 one-frame calls (every sweep complete)
    bit for bit, with the ship pushing into the ice edge."""
    from mbd_icenav_b200 import rollouts, scene
    from mbd_icenav_b200.sim import build_sim_context
    from mbd_icenav_b200.state import build_initial_ice_state, build_initial_ship_state
    f = scene.make_medium_field(seed=2, n_frames=40)
    K = 40
    eta0 = rollouts.ice_edge_pose(f, gap=0.5)
    d = np.array([np.cos(eta0[2]), np.sin(eta0[2])])
    path = np.array([[eta0[0] + 2.0 * 0.05 * i * d[0], eta0[1] + 2.0 * 0.05 * i * d[1], eta0[2]]
                     for i in range(K + 2)])
    ctx = build_sim_context(f.polygons, f.centroids, f.bonds, eta0[:2], f.ship_length, f.ship_beam, K, f.dt,
                            (0.0, 0.0), f.thicknesses, f.ship_props, parent_ids=f.parent_ids, verbose=False,
                            n_ice_steps=f.n_ice_steps, hull_local=f.hull_local, dilation=0.05,
                            dtype=torch.float32, device="cuda")
    fs = ctx.frame_step
    st0 = build_initial_ice_state(f.n, f.centroids, len(f.bonds), ctx.static.initial_floe_of.cpu().numpy(),
                                  dtype=torch.float32, device="cuda")
    sh0 = build_initial_ship_state(eta0[:2], float(eta0[2]), dtype=torch.float32, device="cuda")
    dev = torch.device("cuda", 0)
    rows = torch.as_tensor(np.concatenate([path[:K], path[1:K + 1]], 1), dtype=torch.float32, device=dev)
    vw = torch.zeros((K, f.n, 2), dtype=torch.float32, device=dev)
    st_a, sh_a, h_a = fs.scan_segment(st0, sh0, rows, vw)
    st, sh = st0, sh0
    hist = []
    for i in range(K):
        st, sh, h = fs.scan_segment(st, sh, rows[i:i + 1], vw[i:i + 1])
        hist.append(h)
    for a, b in zip(st_a, st):
        assert torch.equal(a, b)
    for a, b in zip(sh_a, sh):
        assert torch.equal(a, b)
    for j, ha in enumerate(h_a):
        if ha is not None:
            assert torch.equal(ha, torch.cat([h[j] for h in hist])), j
    assert int(st_a.elem_active.sum()) > 0 and int(st_a.elem_active.sum()) < f.n // 4
    fs.close()
