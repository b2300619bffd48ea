"""Host-side planner logic without a GPU: the mid-transit channel starts."""
import math
from types import SimpleNamespace

import numpy as np
import pytest


def _lattice_field(spacing=3.0, n=120):
    """Square elements on a lattice covering ``n * spacing`` metres a side."""
    xs = (np.arange(n) + 0.5) * spacing
    cx, cy = np.meshgrid(xs, xs, indexing="ij")
    cents = np.stack([cx.ravel(), cy.ravel()], 1)
    h = 0.45 * spacing
    square = np.array([[-h, -h], [h, -h], [h, h], [-h, h]])
    return SimpleNamespace(centroids=cents, polygons=[c + square for c in cents], ship_length=60.0, ship_beam=12.0,
                           dt=0.05, trajectory=np.array([[0.0, -40.0, math.pi / 2]]),
                           domain=(0.0, n * spacing, 0.0, n * spacing))


def test_channel_starts_clear_the_hull_and_the_lane_behind_it():
    from mbd_icenav_b200 import planner
    f = _lattice_field()
    rng = np.random.default_rng(0)
    radii = planner.element_radii(f)
    assert radii == pytest.approx(np.full(len(radii), 0.45 * 3.0 * math.sqrt(2)))
    starts = planner.channel_starts(f, 6, rng, horizon=64, clearance=2.0, channel=100.0)
    R = planner.reach_radius(f, 64, f.dt)
    cents = f.centroids
    for eta, removed in starts:
        x, y, psi = eta
        assert abs(psi - math.pi / 2) <= 0.3
        # the whole reach lies inside the ice
        assert cents[:, 0].min() + R <= x <= cents[:, 0].max() - R
        assert cents[:, 1].min() + R <= y <= cents[:, 1].max() - R
        c, s = math.cos(psi), math.sin(psi)
        dx, dy = cents[:, 0] - x, cents[:, 1] - y
        bx, by = c * dx + s * dy, -s * dx + c * dy
        r = radii + 2.0
        lane = (bx < 30.0 + r) & (bx > -30.0 - 100.0 - r) & (np.abs(by) < 6.0 + r)
        assert set(np.nonzero(lane)[0].tolist()) == set(np.asarray(removed).tolist())
        # ice ahead of the bow and beside the hull stays
        d = np.hypot(dx, dy)
        kept = np.setdiff1d(np.nonzero(d < R)[0], removed)
        assert len(kept) > 300 and (bx[kept] > 30.0).any()


def test_channel_starts_need_a_field_larger_than_one_window():
    from mbd_icenav_b200 import planner
    with pytest.raises(ValueError):
        planner.channel_starts(_lattice_field(n=30), 1, np.random.default_rng(0))


def test_scene_starts_kinds():
    from mbd_icenav_b200 import planner
    f = _lattice_field()
    out = planner.scene_starts(f, "channel", 2, np.random.default_rng(1))
    assert len(out) == 2 and all(len(rem) > 0 for _, rem in out)
    with pytest.raises(ValueError):
        planner.scene_starts(f, "pack", 1, np.random.default_rng(1))


def test_sweep_features_oracle_known_answer():
    """A ship surging along +x at 2 m/s meets one element 10 m ahead: hit at
    the pose whose grown hull box first holds its centroid."""
    from oracle.rollout_oracle import sweep_features
    H, dt = 20, 0.5
    eta0 = np.zeros((1, 3))
    hist = np.zeros((H, 1, 3))
    hist[:, 0, 0] = np.arange(1, H + 1) * 1.0  # 1 m per step
    pos = np.array([[10.0, 0.0], [10.0, 30.0], [11.5, 0.5]])
    radii = np.array([1.0, 1.0, 0.5])
    masses = np.array([1000.0, 500.0, 200.0])
    f = sweep_features(eta0, hist, pos, radii, masses, [0, 1, 0], [1, 2, 2], 5.0, 2.0, dt)[0]
    # element 0: |10 - x| < 6 first at x = 5 (t = 5); element 2: |11.5 - x| < 5.5
    # first at x = 7 (t = 7); element 1 is never within the beam
    vn2 = 2.0 * 4.5 / np.hypot(4.5, 0.5)
    assert f[0] == 2 and f[1] == 1200.0
    assert f[2] == pytest.approx(0.5 * 1200.0 * 4.0)
    assert f[3] == pytest.approx(1000.0 * 2.0 + 200.0 * vn2)
    assert f[4] == pytest.approx(1000.0 * (H + 1 - 5) / (H + 1) + 200.0 * (H + 1 - 7) / (H + 1))
    assert f[5] == pytest.approx(0.5 * 1000.0 * 4.0 + 0.5 * 200.0 * vn2 ** 2)
    assert f[6] == 2 and f[7] == 1  # bonds (0,1), (1,2) cut; (0,2) both hit


def test_screened_selection_splits_the_check_between_band_and_rest():
    """ScreenedScorer.selection on CPU tensors: the top_k lowest predictions,
    then the check drawn from the band below them (deepen) and from the rest,
    disjoint; without a band, the check comes from everything below the top_k."""
    import torch
    from mbd_icenav_b200.planner import ScreenedScorer
    Q, k, r, D = 200, 10, 8, 40
    pred = torch.randperm(Q, generator=torch.Generator().manual_seed(0)).double()
    order = torch.argsort(pred)

    def scorer(deepen):
        return SimpleNamespace(k=k, n_check=r, deepen=deepen, n_band=min(r // 2, deepen),
                               gen=torch.Generator().manual_seed(1))

    top, chk, band = ScreenedScorer.selection(scorer(D), pred)
    assert torch.equal(top, order[:k]) and torch.equal(band, order[k:k + D])
    assert chk.numel() == r and len(set(chk.tolist()) | set(top.tolist())) == k + r
    assert set(chk[:r // 2].tolist()) <= set(band.tolist())
    assert set(chk[r // 2:].tolist()) <= set(order[k + D:].tolist())
    top0, chk0, band0 = ScreenedScorer.selection(scorer(0), pred)
    assert band0 is None and torch.equal(top0, top)
    assert set(chk0.tolist()) <= set(order[k:].tolist()) and chk0.numel() == r
    # the check's measure: how much the best of the others beats the best, relative to it
    beats = ScreenedScorer._beats
    assert beats(torch.tensor(10.0), torch.tensor([12.0, 8.0])) == pytest.approx(0.25)
    assert beats(torch.tensor(10.0), torch.tensor([12.0])) == 0.0
    assert beats(torch.tensor(10.0), torch.tensor([])) == 0.0


def test_within_scene_rank_corr_on_a_synthetic_dataset():
    """The diagnostic ranks each start's candidates on its own: a feature that
    orders the ice terms within every start scores 1 even when the starts'
    levels differ, and a reversed one -1."""
    import torch
    from mbd_icenav_b200 import planner
    from mbd_icenav_b200 import surrogate as S
    H, per, starts = 4, 16, 3
    n = per * starts
    rng = np.random.default_rng(0)
    extra = np.zeros((n, S.N_SHIP + S.N_STEP * H + S.N_SWEEP), np.float32)
    raw = np.zeros((n, 3))
    for s in range(starts):
        v = rng.permutation(per).astype(np.float64) + 100.0 * (starts - s)
        rows = slice(s * per, (s + 1) * per)
        raw[rows, 0] = v
        raw[rows, 1] = v
        raw[rows, 2] = v
        extra[rows, S.N_SHIP + 3 * H] = v - 100.0 * (starts - s) + 7.0 * s  # same order, other level
        extra[rows, S.N_SHIP + 3 * H + 1] = -v                               # reversed
        extra[rows, S.N_SHIP + 2 * H:S.N_SHIP + 3 * H] = rng.random((per, H))
    data = planner.Dataset(None, torch.as_tensor(np.repeat(np.arange(starts), per)), torch.as_tensor(extra),
                           torch.as_tensor(raw), None, (0.0, 1.0))
    rc = planner.within_scene_rank_corr(data)
    assert rc["elements_hit"]["ke"] == pytest.approx(1.0) and rc["mass_hit"]["bonds"] == pytest.approx(-1.0)
    assert abs(rc["path_costmap"]["impulse"]) < 0.6 and set(rc) >= {"bonds_cut", "path_costmap"}
