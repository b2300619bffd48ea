"""Oracle for the per-rollout cost terms (test infrastructure only).

A NumPy float32 restatement of the reference planner's unweighted cost
components, ``_make_raw_components_fn`` (``medea_ice_ship/jax_mbd_planner.py:
569-665``) with its bilinear costmap query ``_make_query`` (``:128-168``), for a
GIVEN pose path: the planner's rollout function is replaced by the path the
DEM rollout produced.  Pinned bit for bit against the reference run under the
NumPy ``jax`` shim (``tests/golden/rollout_cost_golden.npz``,
``tests/golden/make_rollout_cost_golden.py``); the GPU kernel
``dem_rollout_costs`` is checked against it within float32 summation-order
tolerance.  Also the transferred kinetic energy of each system's ice, in
float64.
"""
from __future__ import annotations

import numpy as np

f32 = np.float32


def query(grid, meta, x, y, oob_penalty=1e8):
    """Bilinear costmap value at float32 points (x, y) (jax_mbd_planner.py:128-168)."""
    xo, yo, res = f32(meta["x_origin"]), f32(meta["y_origin"]), f32(meta["resolution"])
    nrows, ncols = int(meta["rows"]), int(meta["cols"])
    cf = (x - xo) / res - f32(0.5)
    rf = (y - yo) / res - f32(0.5)
    r0 = np.floor(rf).astype(np.int32)
    c0 = np.floor(cf).astype(np.int32)
    fr = (rf - r0).astype(f32)
    fc = (cf - c0).astype(f32)
    r0c, r1c = np.clip(r0, 0, nrows - 1), np.clip(r0 + 1, 0, nrows - 1)
    c0c, c1c = np.clip(c0, 0, ncols - 1), np.clip(c0 + 1, 0, ncols - 1)
    oob = np.where((c0 < 0) | (c0 + 1 >= ncols), f32(oob_penalty), f32(0.0))
    one = f32(1)
    val = (grid[r0c, c0c] * (one - fr) * (one - fc) + grid[r0c, c1c] * (one - fr) * fc
           + grid[r1c, c0c] * fr * (one - fc) + grid[r1c, c1c] * fr * fc)
    return (val + oob).astype(f32)


def waypoint_costs(traj, grid, meta, ship_length=0.0, ship_beam=0.0, oob_penalty=1e8):
    """Costmap value of each pose of traj (W, 3): the query at the hull centre
    and its four box corners, maximum, or at the centre alone without a hull
    (jax_mbd_planner.py:616-620)."""
    traj = np.asarray(traj, f32)
    grid = np.asarray(grid, f32)
    if ship_length > 0 and ship_beam > 0:
        hl, hw = float(ship_length) / 2.0, float(ship_beam) / 2.0
        dxb = np.array([0.0, hl, hl, -hl, -hl], f32)
        dyb = np.array([0.0, hw, -hw, hw, -hw], f32)
        c, s = np.cos(traj[:, 2:3]), np.sin(traj[:, 2:3])
        wx = traj[:, 0:1] + c * dxb - s * dyb
        wy = traj[:, 1:2] + s * dxb + c * dyb
        return query(grid, meta, wx, wy, oob_penalty).max(axis=1)
    return query(grid, meta, traj[:, 0], traj[:, 1], oob_penalty)


def raw_components(traj, u_norm, grid, meta, goal_xy, ship_length=0.0, ship_beam=0.0, cost_truncate_y=None,
                   oob_penalty=1e8):
    """[costmap, path length, goal distance, jerk] of one path traj (H+1, 3) with
    normalised controls u_norm (H, 3) (jax_mbd_planner.py:616-663)."""
    traj = np.asarray(traj, f32)
    u_norm = np.asarray(u_norm, f32)
    grid = np.asarray(grid, f32)
    wp = waypoint_costs(traj, grid, meta, ship_length, ship_beam, oob_penalty)
    d = np.diff(traj[:, :2], axis=0)
    seg = np.sqrt(np.sum(d ** 2, axis=1) + f32(1e-8))
    if cost_truncate_y is not None:
        cm = np.maximum.accumulate(traj[:, 1])
        prev = np.concatenate([np.array([-1e9], f32), cm[:-1]])
        mask = (prev < f32(cost_truncate_y)).astype(f32)
        wp = wp * mask
        length = (seg * mask[:-1]).sum()
    else:
        length = seg.sum()
    cost = (f32(0.5) * (wp[:-1] + wp[1:]) * seg).sum()
    W = traj.shape[0]
    t = np.arange(W, dtype=f32)
    disc = np.exp(-t / f32(float(W) / 3.0))
    disc = disc / disc.sum()
    dist = np.sqrt(np.sum((traj[:, :2] - np.asarray(goal_xy, f32)) ** 2, axis=1) + f32(1e-4))
    goal = np.dot(disc, dist)
    du = np.diff(u_norm, axis=0)
    jerk = np.mean(du ** 2)
    return np.array([cost, length, goal, jerk], f32)


def transferred_ke(masses, v0, v1, system_start):
    """(Q,) sum over each system's elements of 0.5 m (|v1|^2 - |v0|^2), float64."""
    m = np.asarray(masses, np.float64)
    a = np.asarray(v0, np.float64)
    b = np.asarray(v1, np.float64)
    e = 0.5 * m * ((b ** 2).sum(1) - (a ** 2).sum(1))
    s = np.asarray(system_start)
    return np.array([e[s[q]:s[q + 1]].sum() for q in range(len(s) - 1)])


def sweep_features(eta0, hist, pos, radii, masses, bond_i, bond_j, half_len, half_beam, dt):
    """What each rigid-ship pose path sweeps through an ice window: (Q, 8)
    float64, the definition ``dem_rollout_sweep_features`` implements (it has
    no reference counterpart; the screening surrogate reads it).  Pose 0 is
    eta0[q], pose t the row hist[t - 1, q].  Element e is hit at the first pose
    whose frame puts its centroid inside the hull box grown by its radius
    (|x| < half_len + r, |y| < half_beam + r); the geometry is float32 and
    unfused (cos and sin of the heading rounded from float64), the sums
    float64.  Columns: elements hit, their mass, sum 0.5 m |v|^2, sum m v_n,
    sum m (H + 1 - t) / (H + 1), sum 0.5 m v_n^2 (v the path's step velocity
    (pose t - pose t-1) / dt, the first step's at t = 0; v_n its component
    towards the centroid, clamped at 0), bonds with one end hit, bonds with
    both ends hit."""
    eta0 = np.asarray(eta0, np.float64)
    hist = np.asarray(hist, np.float64)
    H, Q = hist.shape[0], hist.shape[1]
    P = np.concatenate([eta0[None], hist], 0)  # (H + 1, Q, 3)
    px, py = P[..., 0].astype(f32), P[..., 1].astype(f32)
    cs, sn = np.cos(P[..., 2]).astype(f32), np.sin(P[..., 2]).astype(f32)
    inv = f32(1.0 / dt)
    vx = np.empty_like(px)
    vy = np.empty_like(py)
    vx[1:] = (px[1:] - px[:-1]) * inv
    vy[1:] = (py[1:] - py[:-1]) * inv
    vx[0], vy[0] = vx[1], vy[1]
    ex, ey = np.asarray(pos, np.float64)[:, 0].astype(f32), np.asarray(pos, np.float64)[:, 1].astype(f32)
    r = np.asarray(radii, np.float64).astype(f32)
    m = np.asarray(masses, np.float64).astype(f32).astype(np.float64)
    gl, gw = f32(half_len) + r, f32(half_beam) + r
    out = np.zeros((Q, 8))
    bi, bj = np.asarray(bond_i, np.int64), np.asarray(bond_j, np.int64)
    for q in range(Q):
        dx = ex[None, :] - px[:, q, None]  # (H + 1, n) float32
        dy = ey[None, :] - py[:, q, None]
        bx = cs[:, q, None] * dx + sn[:, q, None] * dy
        by = cs[:, q, None] * dy - sn[:, q, None] * dx
        inside = (np.abs(bx) < gl[None, :]) & (np.abs(by) < gw[None, :])
        hit = inside.any(0)
        t = np.argmax(inside, 0)[hit]
        e = np.nonzero(hit)[0]
        vxe, vye = vx[t, q].astype(np.float64), vy[t, q].astype(np.float64)
        ddx, ddy = dx[t, e].astype(np.float64), dy[t, e].astype(np.float64)
        dd = np.sqrt(ddx * ddx + ddy * ddy)
        vn = np.maximum(0.0, (vxe * ddx + vye * ddy) / np.maximum(dd, 1e-6))
        me = m[e]
        hb = np.zeros(len(ex), bool)
        hb[e] = True
        out[q] = [len(e), me.sum(), (0.5 * me * (vxe * vxe + vye * vye)).sum(), (me * vn).sum(),
                  (me * (H + 1 - t) / (H + 1)).sum(), (0.5 * me * vn * vn).sum(),
                  np.count_nonzero(hb[bi] != hb[bj]), np.count_nonzero(hb[bi] & hb[bj])]
    return out
