"""NumPy restatement of the DPDEM ice-ship frame step (the oracle).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Every function names the reference lines it restates.  Arithmetic is written
in the reference's operation order so that, in float64, results agree with the
reference executed on NumPy to rounding, and in float32 the contact and bond
predicates are evaluated with the same operations.  Scatter-adds use
``np.add.at``, which applies updates in index order.

Precision: every float array is cast to ``dtype`` (float32 or float64) on
entry; scalar constants are Python floats (weakly typed, as in JAX).

Broad phase: the reference evaluates all ``n(n-1)/2`` pairs
(``jax_ice_state.py:212-214``, ``jax_simulation.py:127-164``).  Pairs whose
disks do not overlap contribute exact zeros, so ``pair_mode="grid"`` (the
"restated broad phase") evaluates only pairs closer than ``r_i + r_j`` plus a
margin, found with a uniform grid, in the same lexicographic order; the sums
are bitwise identical to the all-pairs ones.  ``pair_mode="all"`` is the
literal restatement.

Ship contact pass 2 (``jax_geometry.py:435-510``) is vectorised over the
elements whose bounding circle can reach the hull; elements farther away get
pen = 0, which is what every one of their point tests returns.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import NamedTuple, Optional

import numpy as np

_STRESS_CLIP = 1e12          # jax_bond_fracture.py:21
_SIGMA_MIN_FOR_DAMAGE = 1e4  # jax_bond_fracture.py:22
_DELTA_M_MIN_INITIATE = 1e-5 # jax_bond_fracture.py:23
_DAMAGE_RATE_CAP = 0.15      # jax_bond_fracture.py:24


class OState(NamedTuple):
    positions: np.ndarray
    velocities: np.ndarray
    rotations: np.ndarray
    angular_vels: np.ndarray
    submergence: np.ndarray
    bond_intact: np.ndarray
    bond_damage: np.ndarray
    bond_delta_m_0: np.ndarray
    bond_delta_m_max: np.ndarray
    bond_delta_s: np.ndarray
    elem_active: np.ndarray
    dpdem_floe_eligible: np.ndarray


class OShip(NamedTuple):
    eta: np.ndarray
    nu: np.ndarray
    n_actual: np.ndarray
    e_int: np.ndarray


@dataclass
class OParams:
    """Closure constants of ``_make_frame_step`` (``jax_simulation.py:325-361``)
    plus the ``IceProperties`` constants the step reads."""

    half_len: float
    half_beam: float
    n_edge_samples: int
    bond_stiffness_factor: float
    hertz_factor: float
    hertz_exponent: float
    ice_ice_friction: float
    friction_cap: float
    c_d_drag: float
    drag_ref_thickness: float
    linear_drag_factor: float
    drag_coefficient_moment: float
    angular_damping: float
    angular_cap_lo: float
    angular_cap_hi: float
    velocity_clip: float
    vc_ship: tuple
    position_clip: float
    pen_crit_ref: float
    pen_crit_thk_ref: float
    w_contact_cap: float
    w_contact_factor: float
    side_push_factor: float
    submergence_rate: float
    submergence_pen_cap: float
    rise_time_const: float
    effective_strength_collision: float
    max_fracture_thickness: float
    max_ship_ice_force: Optional[float]
    ice_brake_threshold: float
    bond_cohesion: float
    bond_internal_friction: float
    bond_G_c_I: float
    bond_G_c_II: float
    bond_eta_bk: float
    dt: float
    dt_ice: float
    n_ice_steps: int
    use_auto_icenav: bool
    T_n: float
    youngs_modulus: float = 5e9
    water_density: float = 1025.0
    flexural_strength_base: float = 0.3e6


def params_from_config(cfg, ship_length, ship_beam, n_ice_steps, dt, dt_ice,
                       use_auto_icenav, T_n, youngs_modulus=5e9, water_density=1025.0,
                       flexural_strength_base=0.3e6) -> OParams:
    """Read the factory's constants from a config object (``jax_simulation.py:325-361``)."""
    g = lambda name, d=None: getattr(cfg, name, d)
    lo, hi = g("angular_cap")
    mx = g("max_ship_ice_force")
    return OParams(
        half_len=ship_length / 2.0, half_beam=ship_beam / 2.0,
        n_edge_samples=int(g("n_edge_samples", 3)),
        bond_stiffness_factor=g("bond_stiffness_factor"), hertz_factor=g("hertz_factor"),
        hertz_exponent=g("hertz_exponent"), ice_ice_friction=g("ice_ice_friction"),
        friction_cap=g("friction_cap"), c_d_drag=g("c_d_drag"),
        drag_ref_thickness=g("drag_ref_thickness"), linear_drag_factor=g("linear_drag_factor"),
        drag_coefficient_moment=g("drag_coefficient_moment", 0.4),
        angular_damping=g("angular_damping"), angular_cap_lo=lo, angular_cap_hi=hi,
        velocity_clip=float(np.max(np.abs(g("velocity_clip")))),
        vc_ship=tuple(float(v) for v in g("ship_velocity_clip")),
        position_clip=float(g("position_clip_m", 1e4)),
        pen_crit_ref=g("pen_crit_ref"), pen_crit_thk_ref=g("pen_crit_thickness_ref"),
        w_contact_cap=g("w_contact_cap"), w_contact_factor=g("w_contact_radius_factor"),
        side_push_factor=g("side_push_factor"), submergence_rate=g("submergence_rate"),
        submergence_pen_cap=g("submergence_pen_cap"), rise_time_const=g("rise_time_const"),
        effective_strength_collision=g("effective_strength_collision"),
        max_fracture_thickness=g("max_fracture_thickness", 15.0),
        max_ship_ice_force=None if mx is None else float(mx),
        ice_brake_threshold=float(g("ice_brake_threshold", 0.0)),
        bond_cohesion=g("bond_cohesion"), bond_internal_friction=g("bond_internal_friction"),
        bond_G_c_I=g("bond_G_c_I"), bond_G_c_II=g("bond_G_c_II"), bond_eta_bk=g("bond_eta_bk"),
        dt=float(dt), dt_ice=float(dt_ice), n_ice_steps=int(n_ice_steps),
        use_auto_icenav=bool(use_auto_icenav), T_n=float(T_n),
        youngs_modulus=float(youngs_modulus), water_density=float(water_density),
        flexural_strength_base=float(flexural_strength_base))


class Oracle:
    """Frame-step oracle bound to one ice field (static data) and ship.

    ``static`` and ``ship_dyn`` are objects with the reference's
    ``IceStaticData`` / ``ShipDynamicsData`` field names holding NumPy arrays.
    """

    def __init__(self, static, ship_dyn, params: OParams, B_mat, dtype=np.float64,
                 pair_mode: str = "all", pair_margin: float = 0.0):
        self.dt_ = np.dtype(dtype)
        f = lambda a: np.asarray(a, dtype=self.dt_)
        self.p = params
        s = static
        self.polys = f(s.local_polys_padded)
        self.pmask = np.asarray(s.poly_mask, dtype=bool)
        self.masses, self.inertia, self.radii = f(s.masses), f(s.inertia), f(s.radii)
        self.areas, self.thick = f(s.areas), f(s.thicknesses)
        self.bi = np.asarray(s.bond_i, dtype=np.int64)
        self.bj = np.asarray(s.bond_j, dtype=np.int64)
        self.rest, self.bstr = f(s.rest_lengths), f(s.bond_strengths)
        self.sigma_bar = f(s.sigma_bar_bond)
        self.floe_of = np.asarray(s.initial_floe_of, dtype=np.int64)
        self.k_n, self.k_s = float(s.k_n), float(s.k_s)
        self.n = self.masses.shape[0]
        self.hull = f(ship_dyn.ship_hull_local)
        self.M3inv, self.D3 = f(ship_dyn.M3inv), f(ship_dyn.D3)
        self.Kp, self.Kd, self.Ki = f(ship_dyn.Kp), f(ship_dyn.Kd), f(ship_dyn.Ki)
        self.B_pinv, self.n_max = f(ship_dyn.B_pinv), f(ship_dyn.n_max)
        self.B_mat = f(B_mat)
        self.pair_mode = pair_mode
        self.pair_margin = float(pair_margin)
        # when a list: each substep appends its contact set, the pairs (i < j)
        # with overlap > 0 and distance > 1e-6 (jax_simulation.py:127-131)
        self.contact_log = None
        if pair_mode == "all":
            n = self.n
            self._all_i = np.repeat(np.arange(n), np.arange(n - 1, -1, -1))
            self._all_j = np.concatenate([np.arange(i + 1, n) for i in range(n)]) if n else np.zeros(0, int)
        # max vertex radius per element, for the ship-contact cull
        self.vert_r = np.sqrt((np.asarray(s.local_polys_padded, np.float64) ** 2).sum(-1)).max(-1) if self.n else np.zeros(0)
        # ship reach: outline points (pass 2) and the analytic hull box corners (pass 1)
        self.hull_r = max(float(np.sqrt((np.asarray(ship_dyn.ship_hull_local, np.float64) ** 2).sum(-1)).max()),
                          math.hypot(params.half_len, params.half_beam))

    # ── broad phase ─────────────────────────────────────────────────────────
    def candidate_pairs(self, pos):
        """Pairs (i < j) to evaluate, in lexicographic order."""
        if self.pair_mode == "all":
            return self._all_i, self._all_j
        return grid_pairs(np.asarray(pos, np.float64), np.asarray(self.radii, np.float64),
                          self.pair_margin)

    # ── substep forces (jax_simulation.py:63-268) ───────────────────────────
    def bond_forces(self, st: OState):
        """Bond springs with damage softening (``jax_simulation.py:63-108``)."""
        n = self.n
        dt = self.dt_
        forces = np.zeros((n, 2), dt)
        moments = np.zeros(n, dt)
        if self.bi.shape[0] == 0:
            return forces, moments
        bi, bj = self.bi, self.bj
        d = st.positions[bj] - st.positions[bi]
        dist = np.linalg.norm(d, axis=1)
        dist_safe = np.maximum(dist, 1e-10)
        bdir = d / dist_safe[:, None]
        avg_h = (self.thick[bi] + self.thick[bj]) * 0.5
        stiff = self.p.youngs_modulus * avg_h * self.p.bond_stiffness_factor
        stretch = dist - self.rest
        fmag = stiff * stretch * (1.0 - st.bond_damage)
        fvec = bdir * fmag[:, None]
        fvec = np.where(st.bond_intact[:, None], fvec, 0.0).astype(dt)
        act_i, act_j = st.elem_active[bi], st.elem_active[bj]
        ok = (act_i & act_j) | ((~act_i) & (~act_j))
        fvec = fvec * ok[:, None].astype(dt)
        np.add.at(forces, bi, fvec)
        np.add.at(forces, bj, -fvec)
        cross = 0.5 * (d[:, 0] * fvec[:, 1] - d[:, 1] * fvec[:, 0])
        np.add.at(moments, bi, cross)
        np.add.at(moments, bj, -cross)
        return forces, moments

    def contact_terms(self, pos, vel, pi, pj):
        """Per-pair Hertz normal + capped Coulomb friction (``jax_simulation.py:111-164``).

        Returns (d_vec, overlap, f_n_vec, f_t_vec, cross_val) per pair.
        """
        p = self.p
        dt = self.dt_
        d_vec = pos[pj] - pos[pi]
        dist = np.linalg.norm(d_vec, axis=1)
        min_dist = self.radii[pi] + self.radii[pj]
        overlap = np.maximum(min_dist - dist, 0.0)
        overlap = np.where(dist > 1e-6, overlap, 0.0).astype(dt)
        direction = d_vec / np.maximum(dist[:, None], 1e-10)
        with np.errstate(invalid="ignore", over="ignore"):
            f_n_mag = (p.hertz_factor * overlap ** p.hertz_exponent).astype(dt)
        f_n_vec = direction * f_n_mag[:, None]
        has = overlap > 0.0
        v_rel = vel[pj] - vel[pi]
        v_t = v_rel - np.sum(v_rel * direction, axis=1, keepdims=True) * direction
        v_t_mag = np.linalg.norm(v_t, axis=1)
        t_hat = -v_t / np.maximum(v_t_mag[:, None], 1e-10)
        f_t_mag = np.minimum(p.ice_ice_friction * f_n_mag, p.friction_cap).astype(dt)
        f_t_vec = t_hat * f_t_mag[:, None]
        valid_fric = has & (v_t_mag > 1e-6)
        f_t_vec = np.where(valid_fric[:, None], f_t_vec, 0.0).astype(dt)
        f_n_vec = np.where(has[:, None], f_n_vec, 0.0).astype(dt)
        f_on_i = -f_n_vec - f_t_vec
        cross = -(d_vec[:, 0] * f_on_i[:, 1] - d_vec[:, 1] * f_on_i[:, 0])
        cross = np.where(has, cross, 0.0).astype(dt)
        return d_vec, overlap, f_n_vec, f_t_vec, cross

    def ice_ice_forces(self, st: OState, pairs=None):
        n = self.n
        dt = self.dt_
        forces = np.zeros((n, 2), dt)
        moments = np.zeros(n, dt)
        pi, pj = pairs if pairs is not None else self.candidate_pairs(st.positions)
        if len(pi) == 0:
            if self.contact_log is not None:
                self.contact_log.append(set())
            return forces, moments
        _, overlap, f_n, f_t, cross = self.contact_terms(st.positions, st.velocities, pi, pj)
        if self.contact_log is not None:
            has = overlap > 0.0
            self.contact_log.append(set(zip(pi[has].tolist(), pj[has].tolist())))
        np.add.at(forces, pi, -f_n + f_t)
        np.add.at(forces, pj, f_n - f_t)
        np.add.at(moments, pi, 0.5 * cross)
        np.add.at(moments, pj, -0.5 * cross)
        return forces, moments

    def drag(self, st: OState, v_water):
        """Quadratic drag, linear below 1e-6 m/s (``jax_simulation.py:167-192``)."""
        p = self.p
        rho = p.water_density
        a_drag = self.areas * (self.thick / p.drag_ref_thickness)
        v_rel = st.velocities - v_water
        vmag = np.linalg.norm(v_rel, axis=1, keepdims=True)
        vmag_safe = np.maximum(vmag, 1e-12)
        quad = (v_rel / vmag_safe) * (0.5 * rho * p.c_d_drag * a_drag[:, None] * vmag_safe ** 2)
        lin = 0.5 * rho * p.c_d_drag * a_drag[:, None] * p.linear_drag_factor * v_rel
        return np.where(vmag > 1e-6, quad, lin).astype(self.dt_)

    def rot_drag(self, st: OState):
        """Rotational drag ~ r^3 w|w| A_sub (``jax_simulation.py:195-212``)."""
        p = self.p
        rho = p.water_density
        a_sub = self.areas * np.minimum(st.submergence / np.maximum(self.thick, 1e-10), 1.0)
        return (-0.5 * p.drag_coefficient_moment * rho * (self.radii ** 3)
                * st.angular_vels * np.abs(st.angular_vels) * a_sub).astype(self.dt_)

    def integrate(self, st: OState, forces, moments) -> OState:
        """Semi-implicit Euler with clips, NaN sanitising and frozen mask (``jax_simulation.py:215-268``)."""
        p = self.p
        dt = self.dt_
        accel = forces / self.masses[:, None]
        new_vel = np.clip(st.velocities + accel * p.dt_ice, -p.velocity_clip, p.velocity_clip).astype(dt)
        new_pos = st.positions + new_vel * p.dt_ice
        alpha = moments / self.inertia
        new_avel = st.angular_vels * p.angular_damping + alpha * p.dt_ice
        new_avel = np.clip(new_avel, p.angular_cap_lo, p.angular_cap_hi).astype(dt)
        new_rot = st.rotations + new_avel * p.dt_ice
        new_vel = np.where(np.isfinite(new_vel), new_vel, 0.0).astype(dt)
        new_pos = np.where(np.isfinite(new_pos), new_pos, st.positions)
        new_pos = np.clip(new_pos, -p.position_clip, p.position_clip).astype(dt)
        act = st.elem_active
        new_vel = np.where(act[:, None], new_vel, st.velocities)
        new_pos = np.where(act[:, None], new_pos, st.positions)
        new_avel = np.where(act, new_avel, st.angular_vels)
        new_rot = np.where(act, new_rot, st.rotations)
        return st._replace(positions=new_pos.astype(dt), velocities=new_vel.astype(dt),
                           rotations=new_rot.astype(dt), angular_vels=new_avel.astype(dt))

    def substep(self, st: OState, ship_forces, v_water) -> OState:
        """One substep: F = F_bond + F_ice - F_drag + F_ship (``jax_simulation.py:363-395``)."""
        f_b, m_b = self.bond_forces(st)
        f_i, m_i = self.ice_ice_forces(st)
        f_d = self.drag(st, v_water)
        m_r = self.rot_drag(st)
        forces = f_b + f_i - f_d + ship_forces
        moments = m_b + m_i + m_r
        return self.integrate(st, forces, moments)

    # ── ship contact (jax_geometry.py) ──────────────────────────────────────
    def ship_contact(self, pos, rot, ship_x, ship_y, ship_psi):
        """Per-element max-penetration contact (``jax_geometry.py:515-594``)."""
        dt = self.dt_
        n = self.n
        p = self.p
        pen1, nx1, ny1 = self._pass1(pos, rot, ship_x, ship_y, ship_psi)
        pen2 = np.zeros(n, dt); nx2 = np.zeros(n, dt); ny2 = np.zeros(n, dt)
        reach = self.hull_r + self.vert_r + 1e-3
        dist = np.sqrt((np.asarray(pos[:, 0], np.float64) - float(ship_x)) ** 2
                       + (np.asarray(pos[:, 1], np.float64) - float(ship_y)) ** 2)
        cand = np.nonzero(dist <= reach)[0]
        if len(cand):
            a, b, c = self._pass2(pos[cand], rot[cand], self.polys[cand], self.pmask[cand],
                                  ship_x, ship_y, ship_psi)
            pen2[cand], nx2[cand], ny2[cand] = a, b, c
        use2 = pen2 > pen1
        return (np.where(use2, pen2, pen1).astype(dt), np.where(use2, nx2, nx1).astype(dt),
                np.where(use2, ny2, ny1).astype(dt))

    def _world_verts(self, pos, rot, polys):
        c = np.cos(rot)
        s = np.sin(rot)
        vx, vy = polys[:, :, 0], polys[:, :, 1]
        wx = c[:, None] * vx - s[:, None] * vy + pos[:, 0:1]
        wy = s[:, None] * vx + c[:, None] * vy + pos[:, 1:2]
        return wx.astype(self.dt_), wy.astype(self.dt_)

    def _pass1(self, pos, rot, sx, sy, spsi):
        """Ice vertices + edge samples vs the analytic hull (``jax_geometry.py:139-285``, ``:42-134``)."""
        dt = self.dt_
        p = self.p
        n, V = self.polys.shape[0], self.polys.shape[1]
        wx, wy = self._world_verts(pos, rot, self.polys)
        K = p.n_edge_samples
        if K == 0:
            px, py, pm = wx, wy, self.pmask
        else:
            t = np.linspace(1.0 / (K + 1), K / (K + 1), K).astype(dt)
            nxv, nyv = np.roll(wx, -1, axis=1), np.roll(wy, -1, axis=1)
            ex = wx[:, :, None] * (1.0 - t)[None, None, :] + nxv[:, :, None] * t[None, None, :]
            ey = wy[:, :, None] * (1.0 - t)[None, None, :] + nyv[:, :, None] * t[None, None, :]
            px = np.concatenate([wx[:, :, None], ex], axis=2).reshape(n, V * (1 + K))
            py = np.concatenate([wy[:, :, None], ey], axis=2).reshape(n, V * (1 + K))
            pm = np.repeat(self.pmask, 1 + K, axis=1)
        pen, nx, ny = hull_point_test(px.ravel(), py.ravel(), sx, sy, spsi, p.half_len,
                                      p.half_beam, dt)
        pen = np.where(pm.ravel(), pen, 0.0).astype(dt).reshape(n, -1)
        nx = nx.reshape(n, -1)
        ny = ny.reshape(n, -1)
        best = np.argmax(pen, axis=1)
        idx = np.arange(n)
        return pen[idx, best], nx[idx, best], ny[idx, best]

    def _pass2(self, pos, rot, polys, pmask, sx, sy, spsi):
        """Hull outline points inside each ice polygon (``jax_geometry.py:300-510``)."""
        dt = self.dt_
        wx, wy = self._world_verts(pos, rot, polys)          # (m, V)
        ch, sh = np.cos(spsi), np.sin(spsi)
        R = np.array([[ch, -sh], [sh, ch]], dtype=dt)
        hull_w = (self.hull @ R.T + np.array([sx, sy], dtype=dt)).astype(dt)  # (S, 2)
        hx, hy = hull_w[:, 0], hull_w[:, 1]
        m = wx.shape[0]
        # masked vertex mean (used to orient edge normals outward)
        n_real = np.maximum(np.sum(pmask.astype(dt), axis=1), 1.0).astype(dt)
        cxc = (np.sum(np.where(pmask, wx, 0.0).astype(dt), axis=1) / n_real).astype(dt)
        cyc = (np.sum(np.where(pmask, wy, 0.0).astype(dt), axis=1) / n_real).astype(dt)
        xi, yi = wx, wy
        xj, yj = np.roll(wx, -1, axis=1), np.roll(wy, -1, axis=1)
        # ray-casting PIP, (m, S, V)
        P_x = hx[None, :, None]
        P_y = hy[None, :, None]
        XI, XJ = xi[:, None, :], xj[:, None, :]
        YI, YJ = yi[:, None, :], yj[:, None, :]
        cond_y = (YI > P_y) != (YJ > P_y)
        with np.errstate(divide="ignore", invalid="ignore"):
            x_int = (XJ - XI) * (P_y - YI) / (YJ - YI + 1e-10) + XI
        crosses = cond_y & (P_x < x_int)
        inside = np.sum(crosses.astype(np.int32), axis=2) % 2 == 1       # (m, S)
        # distance to each edge
        vx_, vy_ = XJ - XI, YJ - YI
        wx_, wy_ = P_x - XI, P_y - YI
        c1 = wx_ * vx_ + wy_ * vy_
        c2 = vx_ * vx_ + vy_ * vy_ + 1e-20
        tt = np.clip(c1 / c2, 0.0, 1.0)
        qx = XI + tt * vx_
        qy = YI + tt * vy_
        dist = np.sqrt((P_x - qx) ** 2 + (P_y - qy) ** 2 + 1e-20).astype(dt)  # (m, S, V)
        # outward edge normals
        ex, ey = xj - xi, yj - yi
        nxe, nye = ey, -ex
        nlen = np.sqrt(nxe ** 2 + nye ** 2 + 1e-20)
        nxe, nye = nxe / nlen, nye / nlen
        midx, midy = (xi + xj) / 2.0, (yi + yj) / 2.0
        dotc = (midx - cxc[:, None]) * nxe + (midy - cyc[:, None]) * nye
        flip = dotc < 0.0
        nxe = np.where(flip, -nxe, nxe).astype(dt)
        nye = np.where(flip, -nye, nye).astype(dt)
        best_e = np.argmin(dist, axis=2)                                  # (m, S)
        mi = np.arange(m)[:, None]
        si = np.arange(hx.shape[0])[None, :]
        pen_raw = dist[mi, si, best_e]
        nx_b = nxe[mi, best_e]
        ny_b = nye[mi, best_e]
        pen_s = np.where(inside, pen_raw, 0.0).astype(dt)
        nx_s = np.where(inside, nx_b, 0.0).astype(dt)
        ny_s = np.where(inside, ny_b, 0.0).astype(dt)
        best_s = np.argmax(pen_s, axis=1)
        pen_i = pen_s[np.arange(m), best_s]
        nx_i = nx_s[np.arange(m), best_s]
        ny_i = ny_s[np.arange(m), best_s]
        upd = pen_i > 0.0
        return (np.where(upd, pen_i, 0.0).astype(dt), np.where(upd, nx_i, 0.0).astype(dt),
                np.where(upd, ny_i, 0.0).astype(dt))

    # ── frame step (jax_simulation.py:397-699) ──────────────────────────────
    def frame_step(self, st: OState, ship: OShip, setpoint, setpoint_next, v_water,
                   dpdem_eligible, v_water_ship=None, u_ctrl=None):
        """One frame (``jax_simulation.py:397-699``); ``u_ctrl`` (body-frame [X, Y, N])
        drives the ship instead of the setpoints, as planner rollouts do."""
        p = self.p
        dt = self.dt_
        st = OState(*[np.asarray(a, dtype=(bool if np.asarray(a).dtype == bool else dt)) for a in st])
        ship = OShip(*[np.asarray(a, dt) for a in ship])
        setpoint = np.asarray(setpoint, dt)
        setpoint_next = np.asarray(setpoint_next, dt)
        v_water = np.asarray(v_water, dt)
        dpdem_eligible = np.asarray(dpdem_eligible, bool)
        v_water_ship = np.zeros(2, dt) if v_water_ship is None else np.asarray(v_water_ship, dt)
        n = self.n
        sx, sy, spsi = ship.eta[0], ship.eta[1], ship.eta[2]

        # 1. collision detection
        pen, nx, ny = self.ship_contact(st.positions, st.rotations, sx, sy, spsi)
        has = pen > 0.0
        # 2. contact force (jax_simulation.py:434-444)
        w_contact = np.minimum(p.w_contact_factor * self.radii, p.w_contact_cap)
        sigma_f = p.flexural_strength_base * np.sqrt(self.thick)
        f_break = sigma_f * w_contact * self.thick ** 2
        pen_crit = p.pen_crit_ref * (self.thick / p.pen_crit_thk_ref)
        force_mag = f_break * np.minimum(pen / np.maximum(pen_crit, 1e-10), 1.0)
        force_mag = np.where(has, force_mag, 0.0).astype(dt)
        soi_x = force_mag * nx
        soi_y = force_mag * ny
        rel_y = st.positions[:, 1] - sy
        soi_y = soi_y + p.side_push_factor * force_mag * np.sign(rel_y)
        soi = np.stack([soi_x, soi_y], axis=1).astype(dt)
        # thrust cap (jax_simulation.py:459-468)
        if p.max_ship_ice_force is not None:
            tot = np.linalg.norm(np.sum(soi, axis=0))
            scale = np.where(tot > p.max_ship_ice_force,
                             p.max_ship_ice_force / np.maximum(tot, 1e-6), 1.0).astype(dt)
            soi = soi * scale
            force_mag = force_mag * scale
        F_ship = -np.sum(soi, axis=0)
        r_x = st.positions[:, 0] - sx
        r_y = st.positions[:, 1] - sy
        M_ship = np.sum(np.where(has, r_x * (-soi_y) - r_y * (-soi_x), 0.0).astype(dt))
        tau_ice = np.array([F_ship[0], F_ship[1], M_ship], dtype=dt)
        # 3. submergence + buoyancy (jax_simulation.py:478-496)
        pen_c = np.minimum(pen, p.submergence_pen_cap)
        new_sub = np.where(has,
                           np.minimum(st.submergence + p.submergence_rate * pen_c * p.dt, self.thick),
                           np.maximum(0.0, st.submergence - (1.0 / p.rise_time_const) * st.submergence * p.dt)).astype(dt)
        z_sub = np.minimum(new_sub, self.thick)
        f_buoy = p.water_density * 9.81 * self.areas * z_sub
        soi_x = soi_x + np.where(has, f_buoy * nx, 0.0)
        soi_y = soi_y + np.where(has, f_buoy * ny, 0.0)
        soi = np.stack([soi_x, soi_y], axis=1).astype(dt)
        st = st._replace(submergence=new_sub)
        # 4. floe activation (jax_simulation.py:498-509)
        n_floes = dpdem_eligible.shape[0]
        collided = np.zeros(n_floes, np.int32)
        np.maximum.at(collided, self.floe_of, has.astype(np.int32))
        collided = collided.astype(bool)
        new_active = st.elem_active | collided[self.floe_of]
        st = st._replace(elem_active=new_active)
        # 5. eligibility (jax_simulation.py:511-524)
        if self.bi.shape[0] > 0:
            thr = np.min(self.bstr) * p.effective_strength_collision
            fmax = np.zeros(n_floes, dt)
            np.maximum.at(fmax, self.floe_of, force_mag)
            new_elig = dpdem_eligible | (collided & (fmax > thr))
        else:
            new_elig = dpdem_eligible
        # 6. substeps
        for _ in range(p.n_ice_steps):
            st = self.substep(st, soi, v_water)
        # 7. fracture (jax_simulation.py:534-653)
        if self.bi.shape[0] > 0:
            st = self.fracture(st, force_mag, new_active, new_elig)
        st = st._replace(dpdem_floe_eligible=new_elig)
        # 8. ship (jax_simulation.py:655-690)
        if u_ctrl is not None:
            # planner rollouts: controls drive the ship (no setpoints, no ice brake)
            z3 = np.zeros(3, dtype=dt)
            ship_new = self.ship_step(ship, z3, z3, tau_ice, v_water_ship, u_ctrl=u_ctrl)
        elif p.ice_brake_threshold > 0.0:
            surge = np.abs(tau_ice[0])
            bf = np.clip(p.ice_brake_threshold / np.maximum(surge, p.ice_brake_threshold), 0.1, 1.0)
            eff_sp = np.array([ship.eta[0] + bf * (setpoint[0] - ship.eta[0]),
                               ship.eta[1] + bf * (setpoint[1] - ship.eta[1]), setpoint[2]], dtype=dt)
            ship_new = self.ship_step(ship, eff_sp, setpoint_next, tau_ice, v_water_ship)
        else:
            ship_new = self.ship_step(ship, setpoint, setpoint_next, tau_ice, v_water_ship)
        diag = {"pen_max": pen, "force_mag": force_mag,
                "F_ice_on_ship": np.array([F_ship[0], F_ship[1]], dtype=dt),
                "J_cumul_incr": (np.linalg.norm(tau_ice[:2]) * p.dt).astype(dt)}
        return st, ship_new, diag

    def fracture(self, st: OState, force_mag, new_active, new_elig) -> OState:
        """Crack front, DPDEM damage and direct collision breaks (``jax_simulation.py:534-653``)."""
        p = self.p
        dt = self.dt_
        bi, bj = self.bi, self.bj
        n = self.n
        d = st.positions[bj] - st.positions[bi]
        dist = np.linalg.norm(d, axis=1)
        bdir = d / np.maximum(dist, 1e-10)[:, None]
        both_act = new_active[bi] & new_active[bj]
        floe_ok = new_elig[self.floe_of[bi]] & new_elig[self.floe_of[bj]]
        breakable = (self.thick[bi] <= p.max_fracture_thickness) & (self.thick[bj] <= p.max_fracture_thickness)
        near = (force_mag[bi] > 0) | (force_mag[bj] > 0)
        broken = ~st.bond_intact
        crack = np.zeros(n, np.int32)
        np.maximum.at(crack, bi, broken.astype(np.int32))
        np.maximum.at(crack, bj, broken.astype(np.int32))
        crack = crack.astype(bool)
        at_crack = crack[bi] | crack[bj]
        dpdem_ok = both_act & floe_ok & (near | at_crack) & breakable
        v_rel = st.velocities[bj] - st.velocities[bi]
        v_n = np.sum(v_rel * bdir, axis=1)
        v_t = v_rel - v_n[:, None] * bdir
        ds_incr = np.linalg.norm(v_t, axis=1) * p.dt_ice
        ds_gate = near & both_act & floe_ok & breakable
        new_ds = (st.bond_delta_s + np.where(ds_gate, ds_incr, 0.0)).astype(dt)
        L0 = np.maximum(self.rest, 1e-10)
        delta_n = (dist - self.rest).astype(dt)
        delta_n_d = np.where(near, delta_n, 0.0).astype(dt)
        sig_n_el = self.k_n * (delta_n_d / L0)
        sig_t_el = self.k_s * (new_ds / L0)
        sig_n = (sig_n_el * (1.0 - st.bond_damage)).astype(dt)
        sig_t = (sig_t_el * (1.0 - st.bond_damage)).astype(dt)
        nd, nmax, n0, nint = bond_damage_update(
            delta_n, new_ds, sig_n, sig_t, self.sigma_bar, p.bond_cohesion,
            p.bond_internal_friction, p.bond_G_c_I, p.bond_G_c_II, p.bond_eta_bk,
            st.bond_damage, st.bond_delta_m_max, st.bond_delta_m_0, st.bond_intact, dt)
        nd = np.where(dpdem_ok, nd, st.bond_damage)
        nmax = np.where(dpdem_ok, nmax, st.bond_delta_m_max)
        n0 = np.where(dpdem_ok, n0, st.bond_delta_m_0)
        nint_d = np.where(dpdem_ok & breakable, nint, st.bond_intact)
        coll_on = (force_mag[bi] > 0) | (force_mag[bj] > 0)
        coll_f = np.maximum(force_mag[bi], force_mag[bj])
        eff = self.bstr * p.effective_strength_collision
        brk = st.bond_intact & coll_on & (coll_f > eff) & breakable
        final = nint_d & ~brk
        return st._replace(bond_damage=nd.astype(dt), bond_delta_m_max=nmax.astype(dt),
                           bond_delta_m_0=n0.astype(dt), bond_delta_s=new_ds, bond_intact=final)

    def ship_step(self, ship: OShip, setpoint, setpoint_next, tau_ice, v_water_ship, u_ctrl=None) -> OShip:
        e, nu, na, ei = ship_step(ship.eta, ship.nu, ship.n_actual, ship.e_int, setpoint,
                                  setpoint_next, tau_ice, self.M3inv, self.D3, self.Kp, self.Kd,
                                  self.Ki, self.B_pinv, self.n_max, self.B_mat, self.p.T_n,
                                  self.p.dt, v_water_ship, self.p.use_auto_icenav,
                                  self.p.vc_ship, self.dt_, u_ctrl=u_ctrl)
        return OShip(e, nu, na, ei)

    # ── scan (jax_simulation.py:1308-1335) ──────────────────────────────────
    def scan_segment(self, st, ship, setpoints_K6, v_water_Kn2, v_water_ship_K2=None):
        K = setpoints_K6.shape[0]
        hist = {k: [] for k in ("positions", "rotations", "bond_intact", "eta", "submergence",
                                "J", "F_ice_on_ship")}
        for k in range(K):
            vws = None if v_water_ship_K2 is None else v_water_ship_K2[k]
            st, ship, diag = self.frame_step(st, ship, setpoints_K6[k, :3], setpoints_K6[k, 3:],
                                             v_water_Kn2[k], st.dpdem_floe_eligible, vws)
            hist["positions"].append(st.positions)
            hist["rotations"].append(st.rotations)
            hist["bond_intact"].append(st.bond_intact)
            hist["eta"].append(ship.eta)
            hist["submergence"].append(st.submergence)
            hist["J"].append(diag["J_cumul_incr"])
            hist["F_ice_on_ship"].append(diag["F_ice_on_ship"])
        return st, ship, {k: np.stack(v) for k, v in hist.items()}


# ── free functions ──────────────────────────────────────────────────────────

def grid_pairs(pos: np.ndarray, radii: np.ndarray, margin: float = 0.0):
    """All (i < j) with |p_i - p_j| < r_i + r_j + margin, lexicographic order.

    Candidates come from a KD-tree ball query of radius 2 max(r) + margin
    (a superset), then the per-pair test keeps a further rounding margin so
    that every pair the reference's predicate can count is kept.
    """
    from scipy.spatial import cKDTree

    n = pos.shape[0]
    empty = (np.zeros(0, np.int64), np.zeros(0, np.int64))
    if n < 2:
        return empty
    ok = np.isfinite(pos).all(axis=1)
    idx = np.nonzero(ok)[0]
    if len(idx) < 2:
        return empty
    tree = cKDTree(pos[idx])
    pr = tree.query_pairs(r=2.0 * float(radii.max()) + margin + 1e-6, output_type="ndarray")
    if len(pr) == 0:
        return empty
    a, b = idx[pr[:, 0]], idx[pr[:, 1]]
    pi, pj = np.minimum(a, b), np.maximum(a, b)
    d = np.sqrt(((pos[pj] - pos[pi]) ** 2).sum(1))
    keep = d < radii[pi] + radii[pj] + margin + 1e-6 * (1.0 + np.abs(pos[pi]).max(1))
    pi, pj = pi[keep], pj[keep]
    o = np.lexsort((pj, pi))
    return pi[o].astype(np.int64), pj[o].astype(np.int64)


def hull_point_test(px, py, ship_x, ship_y, heading, half_len, half_beam, dt,
                    bow_taper_start: float = 0.6):
    """Points vs the analytic tapered hull, bow at body -x (``jax_geometry.py:42-134``)."""
    c_neg = np.cos(-heading)
    s_neg = np.sin(-heading)
    dx = px - ship_x
    dy = py - ship_y
    rel_x = c_neg * dx - s_neg * dy
    rel_y = s_neg * dx + c_neg * dy
    x_rel = rel_x / half_len
    in_bow = x_rel < -bow_taper_start
    t_bow = np.clip((-x_rel - bow_taper_start) / (1.0 - bow_taper_start), 0.0, 1.0)
    hb_bow = half_beam * (1.0 - 0.9 * t_bow ** 1.5)
    hb_bow = np.maximum(hb_bow, half_beam * 0.05)
    hb = np.where(in_bow, hb_bow, half_beam)
    inside = (rel_x >= -half_len) & (rel_x <= half_len) & (np.abs(rel_y) <= hb)
    d_bow = rel_x + half_len
    d_side = hb - np.abs(rel_y)
    bow_ang = 0.3 + 0.5 * t_bow
    nx_bow = -np.cos(bow_ang)
    ny_bow = np.sign(rel_y) * np.sin(bow_ang)
    pen_bow = np.minimum(d_bow, d_side) + 0.5
    side = d_side <= d_bow
    nx_nb = np.where(side, 0.0, -1.0)
    ny_nb = np.where(side, np.sign(rel_y), 0.0)
    pen_nb = np.where(side, d_side, d_bow)
    nx_b = np.where(in_bow, nx_bow, nx_nb)
    ny_b = np.where(in_bow, ny_bow, ny_nb)
    pen_raw = np.where(in_bow, pen_bow, pen_nb)
    c_h = np.cos(heading)
    s_h = np.sin(heading)
    nx_w = c_h * nx_b - s_h * ny_b
    ny_w = s_h * nx_b + c_h * ny_b
    pen = np.where(inside, np.maximum(pen_raw, 0.0), 0.0).astype(dt)
    return pen, np.where(inside, nx_w, 0.0).astype(dt), np.where(inside, ny_w, 0.0).astype(dt)


def bond_damage_update(delta_n, delta_s, sigma_n, sigma_t, sigma_bar, C, mu_b, G_c_I, G_c_II,
                       eta_bk, cur_damage, cur_dm_max, cur_dm_0, intact, dt):
    """Hybrid criterion, Mohr-Coulomb, damage variable, BK energy (``jax_bond_fracture.py:29-208``)."""
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        delta_n = np.clip(delta_n, -1e3, 1e3)
        delta_s = np.clip(delta_s, -1e3, 1e3)
        sigma_bar = np.clip(sigma_bar, 1e-10, _STRESS_CLIP)
        # equivalent deformation (:69-77)
        dn = np.clip(delta_n, -1e3, 1e3)
        ds = np.clip(np.abs(delta_s), 0.0, 1e3)
        dnp = np.maximum(dn, 0.0)
        delta_m = np.sqrt(np.clip(dnp ** 2 + ds ** 2 + 1e-20, 0.0, 1e12)).astype(dt)
        new_max = np.maximum(cur_dm_max, delta_m)
        # Mohr-Coulomb (:60-66) and strength criterion (:35-57)
        tau_bar = np.maximum(C - mu_b * sigma_n, 1e-6).astype(dt)
        s_pos = np.maximum(np.clip(sigma_n, -_STRESS_CLIP, _STRESS_CLIP), 0.0)
        tau = np.clip(sigma_t, -_STRESS_CLIP, _STRESS_CLIP)
        sb = np.maximum(np.clip(sigma_bar, 1e-10, _STRESS_CLIP), 1e-10)
        tb = np.maximum(np.clip(tau_bar, 1e-10, _STRESS_CLIP), 1e-10)
        crit = np.clip((s_pos / sb) ** 2 + (tau / tb) ** 2, 0.0, 1e10).astype(dt)
        initiating = (crit >= 1.0) & (cur_dm_0 <= 0.0) & (delta_m > _DELTA_M_MIN_INITIATE)
        new_0 = np.where(initiating, delta_m, cur_dm_0).astype(dt)
        # energy ratio and BK (:103-121)
        dnp2 = np.maximum(delta_n, 0.0)
        g_ratio = (delta_s ** 2 / (dnp2 ** 2 + 1e-10)).astype(dt)
        g_I = 1.0 / (1.0 + g_ratio + 1e-10)
        g_II = g_ratio / (1.0 + g_ratio + 1e-10)
        g_tot = g_I + g_II + 1e-10
        ratio = g_II / g_tot
        g_c = (G_c_I + (G_c_II - G_c_I) * np.power(ratio, eta_bk)).astype(dt)
        s_n_c = np.clip(sigma_n, -_STRESS_CLIP, _STRESS_CLIP)
        s_t_c = np.clip(sigma_t, -_STRESS_CLIP, _STRESS_CLIP)
        sm0_raw = np.sqrt(np.clip(np.maximum(s_n_c, 0.0) ** 2 + s_t_c ** 2 + 1e-20, 0.0, 1e24)).astype(dt)
        sm0 = np.maximum(sm0_raw, 1e-10)
        dm_f = (2.0 * g_c / (np.abs(sm0) + 1e-10)).astype(dt)
        meaningful = sm0_raw >= _SIGMA_MIN_FOR_DAMAGE
        has_dmg = (new_0 > 0.0) & meaningful
        # damage variable (:80-100)
        dmc = np.clip(delta_m, 0.0, 1e6)
        d0c = np.clip(new_0, 0.0, 1e6)
        dfc = np.maximum(np.clip(dm_f, 1e-10, 1e6), 1e-10)
        dmaxc = np.maximum(np.clip(new_max, 0.0, 1e6), d0c + 1e-10)
        denom = np.maximum(dmaxc * (dfc - d0c + 1e-10), 1e-20)
        D = np.clip(dfc * (dmaxc - d0c) / denom, 0.0, 1.0).astype(dt)
        comp = np.where(has_dmg, D, cur_damage)
        new_d = np.where(meaningful, np.maximum(comp, cur_damage), cur_damage)
        new_d = np.minimum(new_d, cur_damage + _DAMAGE_RATE_CAP).astype(dt)
        new_int = intact & (new_d < 1.0)
    return new_d, new_max.astype(dt), new_0, new_int


def ship_step(eta, nu, n_actual, e_int, setpoint, setpoint_next, tau_ice, M3inv, D3, Kp, Kd, Ki,
              B_pinv, n_max, B, T_n, dt_f, v_water_ship, use_auto, vc, dt, u_ctrl=None):
    """DP pole placement + feed-forward, allocation, propeller lag, Fossen Euler
    (``jax_vessel_dynamics.py:246-348`` with ``:54-84``, ``:127-228``, ``:233-243``).

    With ``u_ctrl`` (body-frame [X, Y, N]) the control replaces the controller and
    the allocation, as planner rollouts compose ``ship_euler_step_jax`` with the ice
    force; RPMs and the integral error are kept."""
    pi = math.pi
    psi = eta[2]
    c, s = np.cos(psi), np.sin(psi)
    R = np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]], dtype=dt)
    nu_c = (R.T @ np.array([v_water_ship[0], v_water_ship[1], 0.0], dtype=dt)).astype(dt)
    tau_ice_b = (R.T @ tau_ice).astype(dt)
    if u_ctrl is not None:
        return _euler_clip(eta, nu, np.asarray(u_ctrl, dt) + tau_ice_b, nu_c, M3inv, D3, dt_f, vc, dt) + (
            np.asarray(n_actual, dt), np.asarray(e_int, dt))
    dpsi_d = (setpoint_next[2] - setpoint[2] + pi) % (2.0 * pi) - pi
    v_d = np.array([(setpoint_next[0] - setpoint[0]) / dt_f,
                    (setpoint_next[1] - setpoint[1]) / dt_f, dpsi_d / dt_f], dtype=dt)
    nu_d = (R.T @ v_d).astype(dt)
    tau_ff = ((D3 + Kd) @ nu_d).astype(dt)
    # dp_control (jax_vessel_dynamics.py:127-184)
    e_xy = eta[:2] - setpoint[:2]
    e_psi = (eta[2] - setpoint[2] + pi) % (2.0 * pi) - pi
    e = np.array([e_xy[0], e_xy[1], e_psi], dtype=dt)
    tau_c = (-(R.T @ Kp @ e) - (Kd @ nu) - (R.T @ Ki @ e_int)).astype(dt)
    e_int_new = (e_int + dt_f * e).astype(dt)
    if use_auto:
        u = B_pinv @ (tau_c + tau_ff)
        n_cmd = np.sign(u) * np.sqrt(np.abs(u) + 1e-12)
        n_cmd = np.clip(n_cmd, -n_max, n_max)
        na_new = (n_actual + dt_f * (n_cmd - n_actual) / T_n).astype(dt)
        tau_act = (B @ (np.abs(na_new) * na_new)).astype(dt)
    else:
        tau_act = (tau_c + tau_ff).astype(dt)
        na_new = n_actual
    tau_tot = (tau_act + tau_ice_b).astype(dt)
    return _euler_clip(eta, nu, tau_tot, nu_c, M3inv, D3, dt_f, vc, dt) + (np.asarray(na_new, dt), e_int_new)


def _euler_clip(eta, nu, tau_tot, nu_c, M3inv, D3, dt_f, vc, dt):
    """Fossen Euler step and velocity clip (``jax_vessel_dynamics.py:54-84``, ``:233-243``)."""
    pi = math.pi
    psi = eta[2]
    tau_tot = np.asarray(tau_tot, dt)
    # Euler (jax_vessel_dynamics.py:54-84)
    nu_r = nu - nu_c
    nu_dot = M3inv @ (tau_tot - D3 @ nu_r)
    nu_new = (nu + dt_f * nu_dot).astype(dt)
    cp, sp = np.cos(psi), np.sin(psi)
    vx = cp * nu_new[0] - sp * nu_new[1]
    vy = sp * nu_new[0] + cp * nu_new[1]
    psi_new = (psi + dt_f * nu_new[2] + pi) % (2.0 * pi) - pi
    eta_new = np.array([eta[0] + dt_f * vx, eta[1] + dt_f * vy, psi_new], dtype=dt)
    nu_new = np.array([np.clip(nu_new[0], -vc[0], vc[0]), np.clip(nu_new[1], -vc[1], vc[1]),
                       np.clip(nu_new[2], -vc[2], vc[2])], dtype=dt)
    return eta_new, nu_new
