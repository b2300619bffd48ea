"""The planner pieces on the GPU: the rigid-ship rollout against the oracle's
vessel step, the per-rollout ice terms, shared-window candidate batches, and
the surrogate-screened MBD step (top-k re-scoring and the fallback)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

DEV = torch.device("cuda", 0)


@pytest.fixture(scope="module")
def medium():
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    return bench.load_field("medium", 0)


def _scene(field, eta0=None, dtype=torch.float64):
    from mbd_icenav_b200 import planner, rollouts
    e0 = rollouts.ice_edge_pose(field) if eta0 is None else eta0
    return planner.make_scene(field, e0, (2.0, 0.0, 0.0), horizon=16, dtype=dtype, device=DEV)


def test_ship_rollout_matches_oracle_vessel_step(medium):
    """dem_ship_rollout = the control-driven vessel step with no ice load
    (jax_vessel_dynamics.py:54-84, :233-243), step by step, float64."""
    from mbd_icenav_b200 import planner
    from oracle.dem_oracle import ship_step
    sc = _scene(medium)
    rng = np.random.default_rng(0)
    Q, H = 5, 16
    Yn = torch.as_tensor(rng.uniform(-1, 1, (Q, H, 2)), dtype=torch.float32, device=DEV)
    u = planner.physical_controls(Yn).double()
    comp = planner.rigid_terms(sc, Yn)  # runs dem_ship_rollout
    import ctypes as C
    from mbd_icenav_b200 import _abi
    lib = _abi.load_library()
    eta0 = torch.as_tensor(np.tile(sc.eta0, (Q, 1)), dtype=torch.float64, device=DEV)
    nu0 = torch.as_tensor(np.tile(sc.nu0, (Q, 1)), dtype=torch.float64, device=DEV)
    hist = torch.empty((H, Q, 3), dtype=torch.float64, device=DEV)
    assert lib.dem_ship_rollout(C.byref(sc.params), _abi.DEM_F64, Q, H, eta0.data_ptr(), nu0.data_ptr(),
                                u.data_ptr(), None, hist.data_ptr(), None, None) == 0
    torch.cuda.synchronize()
    P = sc.params
    M3inv = np.array(P.M3inv[:]).reshape(3, 3)
    D3 = np.array(P.D3[:]).reshape(3, 3)
    un = u.cpu().numpy()
    for q in range(Q):
        eta, nu = sc.eta0.copy(), sc.nu0.copy()
        na, ei = np.zeros(6), np.zeros(3)
        for t in range(H):
            eta, nu, na, ei = ship_step(eta, nu, na, ei, np.zeros(3), np.zeros(3), np.zeros(3), M3inv, D3,
                                        np.zeros((3, 3)), np.zeros((3, 3)), np.zeros((3, 3)), np.zeros((6, 3)),
                                        np.ones(6), np.zeros((3, 6)), 1.0, P.dt, np.zeros(2), False,
                                        (P.vc_surge, P.vc_sway, P.vc_yaw), np.float64, u_ctrl=un[t, q])
            np.testing.assert_allclose(hist[t, q].cpu().numpy(), eta, rtol=1e-12, atol=1e-9)
    assert torch.isfinite(comp).all()


def test_shared_window_candidates_equal_their_runs_alone_and_ice_terms(medium):
    """Each candidate of a shared-window batch equals the same candidate run as
    a batch of one, bit for bit; the ice terms are the sums they name."""
    from mbd_icenav_b200 import planner, rollouts
    sc = _scene(medium, dtype=torch.float32)
    w = planner.CostWeights()
    Q = 6
    rng = np.random.default_rng(1)
    Yn = torch.as_tensor(np.clip(rng.normal(0.7, 0.4, (Q, 16, 2)), -1, 1), dtype=torch.float32, device=DEV)
    dem = planner.DemScorer(sc, Q, w)
    terms = dem.terms(Yn)
    u = planner.physical_controls(Yn).to(torch.float32)
    res = rollouts.run(dem.batch, u, history="ship")
    J = res.history[5]  # (H, Q)
    assert torch.allclose(terms[:, 5], J.double().sum(0), rtol=1e-12, atol=0)
    nb = int(dem.batch.bond_start[1].item())
    broken = (dem.batch.state.bond_intact & ~res.state.bond_intact).view(Q, nb).sum(1).double()
    assert torch.equal(terms[:, 6], broken)
    assert (terms[:, 4] >= 0).all() and terms[:, 4].max() > 0, "the candidates must push ice"
    for q in (0, Q - 1):
        one = planner.DemScorer(sc, 1, w)
        t1 = one.terms(Yn[q:q + 1].contiguous())
        assert torch.equal(t1[0], terms[q]), q
        one.batch.frame_step.close()
    dem.batch.frame_step.close()


def test_screened_step_uses_dem_costs_for_top_k_and_falls_back():
    """A surrogate-screened cost batch: the top_k candidates the surrogate ranks
    best and a random check set get their exact DEM costs, every other
    candidate +inf (no unchecked cost can win a step); the step's check is how
    much the best random candidate beats the best screened one; with a
    negative bound every step falls back to the DEM for all candidates (equal
    to the plain DEM batch)."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    from mbd_icenav_b200 import planner
    field = bench.load_field("medium", 0)
    data = planner.generate_dataset(field, n_starts=3, per_start=256, horizon=16, seed=2, device=DEV)
    assert data.extra.shape == (768, 6 + 48 + 8) and torch.isfinite(data.raw).all()
    sur, info = planner.train_surrogate(data, horizon=16, epochs=2, batch=128, device=DEV)
    assert np.isfinite(info["train_loss"][-1])
    sc = planner.make_scene(field, planner.sample_starts(field, 1, np.random.default_rng(9), 16)[0],
                            (2.0, 0.0, 0.0), horizon=16, device=DEV, patch_stats=data.patch_stats)
    w = planner.CostWeights()
    Q, k, r = 256, 16, 8
    rng = np.random.default_rng(3)
    Yn = torch.as_tensor(np.clip(rng.normal(0.7, 0.5, (Q, 16, 2)), -1, 1), dtype=torch.float32, device=DEV)
    plain = planner.DemScorer(sc, Q, w)
    exact = plain(Yn)
    scr = planner.ScreenedScorer(sc, sur, Q, w, top_k=k, n_check=r, max_rel_err=float("inf"), seed=4)
    cost = scr(Yn)
    pred = scr.predicted(Yn)
    top = torch.argsort(pred)[:k]
    kept = torch.isfinite(cost)
    assert int(kept.sum()) == k + r and kept[top].all()
    assert torch.equal(cost[kept], exact[kept])  # the exact DEM costs, as in the full batch
    chk = kept.clone()
    chk[top] = False
    miss = max(0.0, float((exact[top].min() - exact[chk].min()) / exact[chk].min().abs()))
    assert scr.rel_errs[-1] == pytest.approx(miss, rel=1e-12, abs=1e-15) and scr.fallbacks == 0
    fb = planner.ScreenedScorer(sc, sur, Q, w, top_k=k, n_check=r, max_rel_err=-1.0)
    assert torch.equal(fb(Yn), exact) and fb.fallbacks == 1
    # a short plan runs end to end with both cost batches
    cfg = planner.MBDConfig(horizon=16, n_sample=Q, n_diffuse=3, top_k=k)
    Yp, m1 = planner.mbd_plan(plain, cfg, DEV, seed=0)
    Ys, m2 = planner.mbd_plan(scr, cfg, DEV, seed=0)
    assert Yp.shape == (16, 2) and Ys.shape == (16, 2) and len(m1) == len(m2) == 2
    assert np.isfinite(planner.plan_cost(sc, Ys, scr.dem_k))
    # deepening: predictions that put the DEM's best candidates in the band
    # below the top_k and its worst in the top_k; the band's check sample then
    # beats the screened best while the rest cannot beat the band, so the DEM
    # scores the whole band and nothing falls back
    D = 64
    dp = planner.ScreenedScorer(sc, sur, Q, w, top_k=k, n_check=r, max_rel_err=0.0, seed=5, deepen=D)
    order = torch.argsort(exact)  # ascending true cost
    fake = torch.empty_like(exact)
    fake[order[Q - k:]] = torch.arange(k, dtype=fake.dtype, device=DEV)             # worst -> top_k
    fake[order[:D]] = k + torch.arange(D, dtype=fake.dtype, device=DEV)            # best -> band
    fake[order[D:Q - k]] = k + D + torch.arange(Q - k - D, dtype=fake.dtype, device=DEV)
    dp.predicted = lambda Y: fake
    dc = dp(Yn)
    assert dp.deepened == 1 and dp.fallbacks == 0 and dp.band_errs[-1] > 0 and dp.rel_errs[-1] == 0.0
    kept = torch.isfinite(dc)
    assert kept[order[:D]].all() and kept[order[Q - k:]].all()
    assert int(kept.sum()) == k + D + (r - r // 2)  # top_k, the band, the rest's check sample
    assert torch.equal(dc[kept], exact[kept])
    dp.close()


def test_autotune_picks_the_fastest_split_and_caches_it(medium):
    """The work-split autotuner times every choice on the batch, sets the
    fastest, and sets the cached choice for the same bucket without timing;
    the batch's results do not depend on the choice."""
    from mbd_icenav_b200 import autotune, planner, rollouts
    sc = _scene(medium, dtype=torch.float32)
    w = planner.CostWeights()
    Q = 32
    rng = np.random.default_rng(5)
    Yn = torch.as_tensor(np.clip(rng.normal(0.7, 0.4, (Q, 16, 2)), -1, 1), dtype=torch.float32, device=DEV)
    dem = planner.DemScorer(sc, Q, w)
    ref = dem.terms(Yn)
    best, times = dem.autotune(Yn)
    assert set(times) == {c[0] for c in autotune.CHOICES} and best == min(times, key=times.get)
    assert torch.equal(dem.terms(Yn), ref)
    again, t2 = dem.autotune(Yn)
    assert again == best and t2 == {}
    for name, _, _ in autotune.CHOICES:
        autotune.apply(dem.batch.frame_step, name)
        assert torch.equal(dem.terms(Yn), ref), name
    dem.batch.frame_step.close()


def test_channel_scene_leaves_out_the_cleared_elements(medium):
    """A mid-transit scene: the removed elements are in neither the window nor
    the costmap (a max over elements, so no cell rises and some fall), and its
    candidates run."""
    from mbd_icenav_b200 import planner
    (e0, rem), = planner.channel_starts(medium, 1, np.random.default_rng(4), 16)
    sc = planner.make_scene(medium, e0, (2.0, 0.0, 0.0), 16, device=DEV, removed=rem)
    full = planner.make_scene(medium, e0, (2.0, 0.0, 0.0), 16, device=DEV)
    assert len(rem) > 0 and not np.isin(rem, sc.window).any()
    assert set(sc.window.tolist()) == set(full.window.tolist()) - set(rem.tolist())
    assert (sc.costmap.grid <= full.costmap.grid).all() and (sc.costmap.grid < full.costmap.grid).any()
    w = planner.CostWeights()
    Yn = torch.full((4, 16, 2), 0.5, dtype=torch.float32, device=DEV)
    dem = planner.DemScorer(sc, 4, w)
    assert torch.isfinite(dem(Yn)).all()
    dem.batch.frame_step.close()


def test_screened_scorer_adapts_on_dem_scored_candidates_and_restores():
    """With adapt_steps > 0 a step trains the network on the candidates the
    DEM scored (the weights move, the kept costs stay the exact DEM costs) and
    restore() puts back the weights and Adam state bit for bit."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    from mbd_icenav_b200 import planner
    field = bench.load_field("medium", 0)
    data = planner.generate_dataset(field, n_starts=2, per_start=256, horizon=16, seed=3, device=DEV,
                                    scenes="channel")
    sur, _ = planner.train_surrogate(data, horizon=16, epochs=1, batch=128, device=DEV)
    (e0, rem), = planner.channel_starts(field, 1, np.random.default_rng(11), 16)
    sc = planner.make_scene(field, e0, (2.0, 0.0, 0.0), horizon=16, device=DEV, patch_stats=data.patch_stats,
                            removed=rem)
    w = planner.CostWeights()
    Q, k, r = 512, 256, 64
    rng = np.random.default_rng(4)
    Yn = torch.as_tensor(np.clip(rng.normal(0.7, 0.5, (Q, 16, 2)), -1, 1), dtype=torch.float32, device=DEV)
    before = [q.p.clone() for q in sur.net.params()]
    t0 = sur.net.t
    scr = planner.ScreenedScorer(sc, sur, Q, w, top_k=k, n_check=r, max_rel_err=float("inf"), seed=1,
                                 adapt_steps=2)
    cost = scr(Yn)
    kept = torch.isfinite(cost)
    assert int(kept.sum()) == k + r
    exact = planner.DemScorer(sc, Q, w)(Yn)
    assert torch.equal(cost[kept], exact[kept])
    assert sur.net.t == t0 + 2 and any(not torch.equal(a, q.p) for a, q in zip(before, sur.net.params()))
    scr.restore()
    assert sur.net.t == t0 and all(torch.equal(a, q.p) for a, q in zip(before, sur.net.params()))


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_sweep_features_match_oracle(medium, dtype):
    """dem_rollout_sweep_features on the rigid-ship paths of random candidates
    through a real window = the oracle's restatement: counts exact, sums
    within float32 rounding of the float64 totals."""
    from mbd_icenav_b200 import planner
    from oracle.rollout_oracle import sweep_features
    sc = _scene(medium, dtype=dtype)
    rng = np.random.default_rng(3)
    Q, H = 48, 16
    Yn = torch.as_tensor(rng.uniform(-1, 1, (Q, H, 2)), dtype=torch.float32, device=DEV)
    Yn[:, :, 0] = torch.abs(Yn[:, :, 0])  # forward: most paths reach ice
    u = planner.physical_controls(Yn).to(dtype)
    import ctypes as C
    from mbd_icenav_b200 import _abi
    lib = _abi.load_library()
    eta0 = torch.as_tensor(np.tile(sc.eta0, (Q, 1)), dtype=dtype, device=DEV)
    nu0 = torch.as_tensor(np.tile(sc.nu0, (Q, 1)), dtype=dtype, device=DEV)
    hist = torch.empty((H, Q, 3), dtype=dtype, device=DEV)
    rc = lib.dem_ship_rollout(C.byref(sc.params), _abi.DEM_F64 if dtype == torch.float64 else _abi.DEM_F32, Q, H,
                              eta0.data_ptr(), nu0.data_ptr(), u.data_ptr(), None, hist.data_ptr(), None, None)
    assert rc == _abi.DEM_OK
    got = planner.sweep_features(sc, eta0, hist).cpu().numpy().astype(np.float64)
    w = planner.sweep_inputs(sc)
    ref = sweep_features(eta0.cpu().numpy(), hist.cpu().numpy(), w.pos.cpu().numpy(), w.radii.cpu().numpy(),
                         w.masses.cpu().numpy(), w.bi.cpu().numpy(), w.bj.cpu().numpy(),
                         0.5 * medium.ship_length, 0.5 * medium.ship_beam, medium.dt)
    assert (ref[:, 0] > 0).sum() >= Q // 2, "most candidate paths must sweep ice"
    for k in (0, 6, 7):
        np.testing.assert_array_equal(got[:, k], ref[:, k])
    np.testing.assert_allclose(got, ref, rtol=1e-6, atol=0)
    # the same paths again: identical bits (fixed-order sums)
    again = planner.sweep_features(sc, eta0, hist).cpu().numpy().astype(np.float64)
    np.testing.assert_array_equal(again, got)
    # the rigid-path features the screening reads carry them
    _, wcost, sweep = planner.rigid_path(sc, Yn)
    ext = planner.features(sc, Yn, wcost, sweep)
    assert ext.shape == (Q, 6 + 3 * H + 8)
    np.testing.assert_allclose(ext[:, -8:].cpu().numpy(),
                               np.log1p(np.maximum(sweep.cpu().numpy(), 0) / np.array(planner.SWEEP_SCALE)),
                               rtol=1e-5, atol=1e-6)
