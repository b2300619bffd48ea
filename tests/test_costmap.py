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
CASES = ("rand", "nomass", "empty", "window", "nan")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLDEN)


def _case(g, name):
    kw = {}
    for k in ("resolution", "margin", "base_cost", "collision_cost", "obs_cost_buffer_factor", "ship_length",
              "ship_beam", "planning_clearance_margin", "ship_speed", "ship_mass", "ke_cost_scale"):
        v = float(g[f"{name}_{k}"])
        kw[k] = None if np.isnan(v) else v
    bounds = [float(g[f"{name}_{k}"]) for k in ("x_min", "x_max", "y_min", "y_max")]
    masses = g[f"{name}_masses"] if bool(g[f"{name}_has_masses"]) else None
    return g[f"{name}_centroids"], g[f"{name}_thicknesses"], g[f"{name}_radii"], bounds, masses, kw


def _assert_same_grid(got, want, name):
    assert got.shape == want.shape, name
    np.testing.assert_array_equal(np.isnan(got), np.isnan(want), err_msg=name)
    ok = ~np.isnan(want)
    np.testing.assert_array_equal(got[ok], want[ok], err_msg=name)


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_grid(gold, name):
    cents, thick, radii, bounds, masses, kw = _case(gold, name)
    grid, geo = co.build_costmap(cents, thick, radii, *bounds, masses=masses, **kw)
    for k in ("rows", "cols"):
        assert geo[k] == int(gold[f"{name}_res_{k}"])
    for k in ("x_origin", "y_origin", "width", "height"):
        assert geo[k] == float(gold[f"{name}_res_{k}"])
    _assert_same_grid(grid, gold[f"{name}_grid"], name)


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
    _assert_same_grid(np.asarray(res.cost_map), gold[f"{name}_grid"], name)
    assert res.rows == int(gold[f"{name}_res_rows"]) and res.cols == int(gold[f"{name}_res_cols"])
    assert bnd["x_origin"] == float(gold[f"{name}_res_x_origin"])
