"""Golden vectors for the per-rollout planner cost terms.

Usage (in a container where the reference is mounted):

    python tests/golden/make_rollout_cost_golden.py --ref /root/reference

Runs the reference's own ``_make_raw_components_fn`` (``medea_ice_ship/
jax_mbd_planner.py:569-665``) under the NumPy ``jax`` shim in float32 mode (the
planner's precision), with its rollout function replaced by a fixed pose path,
so the output is the four raw cost components of that path on a seeded costmap
grid.  Cases cover the hull-corner query and the centre-only query, paths that
leave the grid's x-extent (the out-of-bounds penalty) and the goal-line
truncation.  Output: ``rollout_cost_golden.npz`` (committed).
"""
from __future__ import annotations

import argparse
import importlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

Q, H = 24, 32
ROWS, COLS = 48, 40


def make_inputs():
    rng = np.random.default_rng(5)
    grid = (0.1 + rng.gamma(0.6, 2.0, (ROWS, COLS))).astype(np.float32)
    meta = dict(x_origin=-20.0, y_origin=-30.0, resolution=2.0, rows=ROWS, cols=COLS)
    traj = np.zeros((Q, H + 1, 3), np.float32)
    for q in range(Q):
        x0 = rng.uniform(-10.0, 50.0) if q % 6 else rng.uniform(-30.0, -18.0)  # some start off the x-extent
        y0 = rng.uniform(-25.0, 40.0)
        psi0 = rng.uniform(-np.pi, np.pi)
        v = rng.uniform(0.2, 1.0)
        w = rng.normal(0.0, 0.05)
        p = np.array([x0, y0, psi0])
        for t in range(H + 1):
            traj[q, t] = p
            p = p + np.array([v * np.cos(p[2]), v * np.sin(p[2]), w])
    u_norm = rng.normal(0.0, 0.4, (Q, H, 3)).astype(np.float32)
    goal = np.array([15.0, 55.0], np.float32)
    hull = np.array([[60.0, 12.0] if q % 3 else [0.0, 0.0] for q in range(Q)])
    trunc = np.array([10.0 if q % 4 == 1 else np.nan for q in range(Q)])
    return grid, meta, traj, u_norm, goal, hull, trunc


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True)
    args = ap.parse_args()
    import jaxshim
    jaxshim.load_reference(args.ref, x64=False)
    planner = importlib.import_module("medea_ice_ship.jax_mbd_planner")
    import jax.numpy as jnp
    grid, meta, traj, u_norm, goal, hull, trunc = make_inputs()
    center = np.array([1e6, 0.0, 0.0], np.float32)
    scale = np.array([1e6, 5e5, 5e8], np.float32)
    out = np.zeros((Q, 4), np.float32)
    for q in range(Q):
        path = jnp.array(traj[q])
        fn = planner._make_raw_components_fn(
            jnp.array(grid), meta, goal, lambda e, n, u, p=path: p, jnp.array(traj[q, 0]), jnp.zeros(3),
            jnp.array(center), jnp.array(scale), ship_length=float(hull[q, 0]), ship_beam=float(hull[q, 1]),
            cost_truncate_y=None if np.isnan(trunc[q]) else float(trunc[q]))
        out[q] = np.asarray(fn(jnp.array(u_norm[q])), np.float32)
    np.savez_compressed(os.path.join(HERE, "rollout_cost_golden.npz"), grid=grid, traj=traj, u_norm=u_norm,
                        goal=goal, hull=hull, trunc=trunc, center=center, scale=scale, raw=out,
                        meta=np.array([meta["x_origin"], meta["y_origin"], meta["resolution"], meta["rows"],
                                       meta["cols"]]))
    print("rollout cost golden:", Q, "paths; oob cases:", int((out[:, 0] >= 1e8).sum()))


if __name__ == "__main__":
    main()
