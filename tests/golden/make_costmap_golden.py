"""Golden vectors for the KE costmap, made by running the reference's own code.

Usage (in a container where the reference is mounted):

    python tests/golden/make_costmap_golden.py --ref /root/reference

The NumPy ``jax`` shim (``jaxshim.py``) is installed in float64 mode, which is
how the reference's costmap tests run (``test_jax_costmap.py:23``), and the
unmodified ``medea_ice_ship/jax_costmap.py`` is imported and called through its
public functions ``build_costmap_jax`` and ``build_costmap_jax_from_ice_state``.
In that mode the rasteriser's float arguments stay double (weakly typed) and
meet the float32 arrays as float32, as JAX's traced weak scalars do.

Cases (inputs and the resulting grid are stored per case in
``costmap_golden.npz``, committed; the tests never need the reference):

* ``rand``   : 60 random elements, masses given, ship 60 x 12 m (7 x 7 dilation);
* ``nomass`` : the same elements, masses from the disk formula, no ship, 1.5 m cells,
               buffer factor 0.3;
* ``empty``  : no elements (open-water grid), with dilation;
* ``window`` : the 500-element medium-field window of the DEM goldens, with its
               reference-built radii / thicknesses / masses, through
               ``build_costmap_jax_from_ice_state``;
* ``nan``    : one element with a NaN centroid (the whole grid becomes NaN);
* ``sic1``   : the ``rand`` elements with the SIC modulation at weight 1.0;
* ``sic_half``: the same elements, masses from the disk formula, 1 m cells, no
               ship, SIC modulation at weight 0.5.
"""
from __future__ import annotations

import argparse
import importlib
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

CASE_KEYS = ("x_min", "x_max", "y_min", "y_max", "resolution", "margin", "base_cost", "collision_cost",
             "obs_cost_buffer_factor", "ship_length", "ship_beam", "planning_clearance_margin",
             "ship_speed", "ship_mass", "ke_cost_scale", "ice_resistance_weight")


def _load_costmap(ref_root: str):
    import jaxshim
    jaxshim.install(True)
    pkg = types.ModuleType("medea_ice_ship")
    pkg.__path__ = [os.path.join(ref_root, "medea_ice_ship")]
    sys.modules["medea_ice_ship"] = pkg
    return importlib.import_module("medea_ice_ship.jax_costmap")


def _cases():
    rng = np.random.default_rng(7)
    n = 60
    cents = np.stack([rng.uniform(0.0, 120.0, n), rng.uniform(0.0, 200.0, n)], 1)
    radii = rng.uniform(0.8, 6.0, n)
    thick = rng.choice([0.5, 1.0, 1.5], n)
    masses = np.pi * radii ** 2 * thick * 900.0 * rng.uniform(0.8, 1.2, n)
    base = dict(x_min=0.0, x_max=120.0, y_min=0.0, y_max=200.0, resolution=2.0, margin=20.0, base_cost=0.1,
                collision_cost=5.0, obs_cost_buffer_factor=0.1, ship_length=60.0, ship_beam=12.0,
                planning_clearance_margin=0.0, ship_speed=4.0, ship_mass=23e6, ke_cost_scale=1e-6,
                ice_resistance_weight=0.0)
    yield "rand", cents, radii, thick, masses, dict(base)
    yield "nomass", cents, radii, thick, None, dict(base, resolution=1.5, obs_cost_buffer_factor=0.3,
                                                    ship_length=None, ship_beam=None, margin=10.0)
    yield "empty", np.zeros((0, 2)), np.zeros(0), np.zeros(0), np.zeros(0), dict(base, margin=5.0)
    g = np.load(os.path.join(HERE, "golden_f64.npz"))
    wc = np.asarray(g["window_pos"][0], np.float64)
    lo, hi = wc.min(0), wc.max(0)
    yield ("window", wc, np.asarray(g["window_static_radii"]), np.asarray(g["window_static_thicknesses"]),
           np.asarray(g["window_static_masses"]),
           dict(base, x_min=float(lo[0]), x_max=float(hi[0]), y_min=float(lo[1]), y_max=float(hi[1]),
                planning_clearance_margin=1.5, ship_speed=2.5))
    c2 = cents.copy()
    c2[5] = np.nan
    yield "nan", c2, radii, thick, masses, dict(base, ship_length=None, ship_beam=None)
    # SIC modulation: the weight of the reference's own test (test_jax_ke_cost.py:381), and a fractional one
    yield "sic1", cents, radii, thick, masses, dict(base, ice_resistance_weight=1.0)
    yield "sic_half", cents, radii, thick, None, dict(base, ice_resistance_weight=0.5, ship_length=None,
                                                      ship_beam=None, resolution=1.0)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True)
    args = ap.parse_args()
    cm = _load_costmap(args.ref)
    out = {}
    for name, cents, radii, thick, masses, kw in _cases():
        if name == "window":
            state = types.SimpleNamespace(positions=cents)
            static = types.SimpleNamespace(thicknesses=thick, radii=radii, masses=masses)
            rest = {k: v for k, v in kw.items() if k not in ("x_min", "x_max", "y_min", "y_max")}
            res, bounds = cm.build_costmap_jax_from_ice_state(state, static, kw["x_min"], kw["x_max"],
                                                              kw["y_min"], kw["y_max"], **rest)
        else:
            rest = {k: v for k, v in kw.items() if k not in ("x_min", "x_max", "y_min", "y_max")}
            res, bounds = cm.build_costmap_jax(cents, thick, radii, kw["x_min"], kw["x_max"], kw["y_min"],
                                               kw["y_max"], masses=masses, **rest)
        out[f"{name}_centroids"] = np.asarray(cents, np.float64)
        out[f"{name}_radii"] = np.asarray(radii, np.float64)
        out[f"{name}_thicknesses"] = np.asarray(thick, np.float64)
        out[f"{name}_has_masses"] = np.array(masses is not None)
        out[f"{name}_masses"] = np.asarray(masses if masses is not None else np.zeros(0), np.float64)
        for k in CASE_KEYS:
            v = kw[k]
            out[f"{name}_{k}"] = np.array(np.nan if v is None else float(v))
        out[f"{name}_grid"] = np.asarray(res.cost_map, np.float32)
        for k in ("x_origin", "y_origin", "resolution", "rows", "cols", "width", "height", "base_cost"):
            out[f"{name}_res_{k}"] = np.array(getattr(res, k))
        print(f"{name}: grid {res.rows}x{res.cols}, max {np.nanmax(res.cost_map) if np.isfinite(res.cost_map).any() else 'nan'}")
    np.savez_compressed(os.path.join(HERE, "costmap_golden.npz"), **out)


if __name__ == "__main__":
    main()
