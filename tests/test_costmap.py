"""KE costmap (jax_costmap.py) — oracle vs the reference's golden grids (CPU), and
the CUDA path through the C ABI vs the same grids (GPU).

Both comparisons are bit-exact: every cell is a maximum of float32 values that
the reference computes with a fixed expression, and maxima do not depend on
the order in which contributions arrive.  NaN cells must match as NaN.
"""
import os

import numpy as np
import pytest

from oracle import costmap_oracle as co

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "costmap_golden.npz")
CASES = ("rand", "nomass", "empty", "window", "nan", "sic1", "sic_half")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLDEN)


def _case(g, name):
    kw = {}
    for k in ("resolution", "margin", "base_cost", "collision_cost", "obs_cost_buffer_factor", "ship_length",
              "ship_beam", "planning_clearance_margin", "ship_speed", "ship_mass", "ke_cost_scale",
              "ice_resistance_weight"):
        v = float(g[f"{name}_{k}"])
        kw[k] = None if np.isnan(v) else v
    bounds = [float(g[f"{name}_{k}"]) for k in ("x_min", "x_max", "y_min", "y_max")]
    masses = g[f"{name}_masses"] if bool(g[f"{name}_has_masses"]) else None
    return g[f"{name}_centroids"], g[f"{name}_thicknesses"], g[f"{name}_radii"], bounds, masses, kw


def _assert_same_grid(got, want, name, ulps=0):
    assert got.shape == want.shape, name
    np.testing.assert_array_equal(np.isnan(got), np.isnan(want), err_msg=name)
    ok = ~np.isnan(want)
    if ulps == 0:
        np.testing.assert_array_equal(got[ok], want[ok], err_msg=name)
    else:
        np.testing.assert_array_max_ulp(got[ok], want[ok], maxulp=ulps)


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_grid(gold, name):
    cents, thick, radii, bounds, masses, kw = _case(gold, name)
    grid, geo = co.build_costmap(cents, thick, radii, *bounds, masses=masses, **kw)
    for k in ("rows", "cols"):
        assert geo[k] == int(gold[f"{name}_res_{k}"])
    for k in ("x_origin", "y_origin", "width", "height"):
        assert geo[k] == float(gold[f"{name}_res_{k}"])
    _assert_same_grid(grid, gold[f"{name}_grid"], name)


def test_sic_box_mean_is_scipys_uniform_filter():
    """The oracle's restated box mean equals SciPy's uniform_filter (mode
    "reflect") bit for bit, which the reference calls (jax_costmap.py:273-278)."""
    from scipy.ndimage import uniform_filter
    rng = np.random.default_rng(3)
    for rows, cols in ((37, 52), (120, 80), (9, 300)):
        occ = (rng.random((rows, cols)) < 0.45).astype(np.float64)
        k = co.sic_window(rows, cols)
        a = np.stack([co.box_mean_1d(occ[:, c], k) for c in range(cols)], 1)
        b = np.stack([co.box_mean_1d(a[r, :], k) for r in range(rows)], 0)
        np.testing.assert_array_equal(b, uniform_filter(occ, size=k, mode="reflect"))


def test_sic_lowers_isolated_floe_cost(gold):
    """The reference's own SIC property (test_jax_ke_cost.py:329-390): the
    modulation lowers the peak cost of sparse ice and never raises a cell."""
    cents, thick, radii, bounds, masses, kw = _case(gold, "sic1")
    plain, _ = co.build_costmap(cents, thick, radii, *bounds, masses=masses, **dict(kw, ice_resistance_weight=0.0))
    sic, _ = co.build_costmap(cents, thick, radii, *bounds, masses=masses, **kw)
    assert sic.max() < plain.max()
    assert np.all(sic <= plain)


def test_reference_properties_hold_on_the_oracle(gold):
    """Properties the reference's own costmap tests check (test_jax_costmap.py):
    open water is the base cost, ice raises the cost, dilation never lowers it."""
    cents, thick, radii, bounds, masses, kw = _case(gold, "rand")
    no_dil, _ = co.build_costmap(cents, thick, radii, *bounds, masses=masses, **dict(kw, ship_beam=None))
    assert np.isclose(no_dil.min(), np.float32(kw["base_cost"]))
    assert no_dil.max() > 10 * kw["base_cost"]
    with_dil, _ = co.build_costmap(cents, thick, radii, *bounds, masses=masses, **kw)
    assert np.all(with_dil >= no_dil)
    assert (with_dil > no_dil).any()


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_cuda_costmap_matches_reference_grid(gold, name):
    torch = pytest.importorskip("torch")
    from mbd_icenav_b200 import costmap
    cents, thick, radii, bounds, masses, kw = _case(gold, name)
    res, bnd = costmap.build_costmap_jax(cents, thick, radii, *bounds, masses=masses, **kw)
    # a fractional SIC weight goes through the reference's float32 power (the C
    # library's powf, within one unit in the last place); the device raises in
    # double and rounds once, so those cells may differ by one unit
    w = kw.get("ice_resistance_weight") or 0.0
    _assert_same_grid(np.asarray(res.cost_map), gold[f"{name}_grid"], name, ulps=0 if w in (0.0, 1.0) else 1)
    assert res.rows == int(gold[f"{name}_res_rows"]) and res.cols == int(gold[f"{name}_res_cols"])
    assert bnd["x_origin"] == float(gold[f"{name}_res_x_origin"])
