"""Chunked simulation driver with device-resident histories.

``simulate_jax_chunked_replan`` mirrors the reference's driver of the same
name (``medea_ice_ship/jax_simulation.py:1438-1796``): same arguments, same
chunk loop (replan callback at every chunk boundary, setpoints from the
trajectory, a current model sampled per frame at the chunk-start positions,
the last short chunk padded to the chunk length and run in full, goal checks
at chunk boundaries) and the same return tuple.

What differs is where the histories live.  The reference downloads every
chunk's full history and appends it frame by frame in Python
(``:1662-1684``); here every frame's positions, rotations, bond masks and
submergence stay in preallocated device buffers, and per chunk only the ship
poses (K x 3 numbers) come to the host, for the goal check; ship poses,
forces and impulses (a few numbers per frame) are downloaded once at the end.
The returned history lists are ``DeviceHistory`` sequences: indexing one
downloads that frame, ``.tensor`` is the whole (frames, ...) device tensor.
"""
from __future__ import annotations

from typing import Optional, Sequence

import numpy as np

from .sim import build_sim_context
from .state import build_initial_ice_state, build_initial_ship_state


class DeviceHistory(Sequence):
    """Per-frame history kept on the device; ``h[f]`` downloads frame f as NumPy."""

    def __init__(self, tensor, length: int):
        self.tensor = tensor
        self._len = int(length)

    def __len__(self):
        return self._len

    def __getitem__(self, i):
        if isinstance(i, slice):
            return [self[j] for j in range(*i.indices(self._len))]
        if i < 0:
            i += self._len
        if not 0 <= i < self._len:
            raise IndexError(i)
        return self.tensor[i].detach().cpu().numpy()

    def to_numpy(self) -> np.ndarray:
        """All frames at once, as one (frames, ...) array."""
        return self.tensor[:self._len].detach().cpu().numpy()


def _trajectory_to_arr(traj) -> np.ndarray:
    if isinstance(traj, (list, tuple)):
        rows = []
        for p in traj:
            if len(p) == 2 and np.ndim(p[0]) > 0:  # ((x, y), heading)
                rows.append([float(p[0][0]), float(p[0][1]), float(p[1])])
            else:
                rows.append([float(p[0]), float(p[1]), float(p[2])])
        return np.asarray(rows, dtype=np.float64).reshape(-1, 3)
    return np.asarray(traj, dtype=np.float64)


def _world_polygons(state, static) -> list:
    """World-frame polygons of the elements (``jax_simulation.py:1405-1435``)."""
    pos = state.positions.detach().cpu().numpy().astype(np.float64)
    rot = state.rotations.detach().cpu().numpy().astype(np.float64)
    polys = np.asarray(static.local_polys_padded.detach().cpu().numpy(), np.float64)
    nv = static.poly_n_verts.detach().cpu().numpy()
    out = []
    for i in range(len(pos)):
        c, s = np.cos(rot[i]), np.sin(rot[i])
        lp = polys[i, :int(nv[i])]
        out.append(np.stack([c * lp[:, 0] - s * lp[:, 1] + pos[i, 0], s * lp[:, 0] + c * lp[:, 1] + pos[i, 1]], 1))
    return out


def simulate_jax_chunked_replan(polygons, centroids, bonds, ship_pos, ship_length, ship_beam, n_frames, dt,
                                drift_vel, thicknesses, ship_props, ship_trajectory=None,
                                return_ship_diagnostics: bool = False, config=None, replan_every_n_frames=None,
                                replan_callback=None, frame_callback=None, parent_ids=None, ocean_current=None,
                                goal_point=None, goal_y_line=None, goal_tolerance: float = 15.0,
                                use_auto_icenav_ship: bool = False, skip_polygon_extraction: bool = False,
                                verbose: bool = True, **context_kw):
    """Receding-horizon simulation in fixed-length scan segments (``jax_simulation.py:1438-1796``).

    ``context_kw`` goes to ``build_sim_context`` (material, dilation, dtype, device, ...).
    Returns ``(positions, rotations, bonds, ship_history, submergence, damage_summary)`` or,
    with ``return_ship_diagnostics``, the diagnostics list in last place.
    """
    import torch

    n = len(polygons)
    chunk = replan_every_n_frames if (replan_every_n_frames and replan_every_n_frames > 0) else n_frames
    ctx = build_sim_context(polygons, centroids, bonds, ship_pos, ship_length, ship_beam, n_frames, dt, drift_vel,
                            thicknesses, ship_props, config=config, parent_ids=parent_ids,
                            use_auto_icenav_ship=use_auto_icenav_ship, chunk_size=chunk, verbose=verbose,
                            **context_kw)
    fs = ctx.frame_step
    dev, dtype = fs.device, fs.dtype
    if ship_trajectory is not None:
        ship_trajectory = _trajectory_to_arr(ship_trajectory)
    start_pos, start_head = np.array(ship_pos, np.float64), 0.0
    if ship_trajectory is not None and len(ship_trajectory) > 0:
        start_pos, start_head = ship_trajectory[0, :2].copy(), float(ship_trajectory[0, 2])
    floe_of = ctx.static.initial_floe_of
    state = build_initial_ice_state(n, centroids, len(bonds), floe_of.detach().cpu().numpy(), dtype=dtype,
                                    device=dev)
    ship_state = build_initial_ship_state(start_pos, start_head, dtype=dtype, device=dev)

    # device history buffers: frame 0 is the initial state (jax_simulation.py:1527-1530)
    F = int(n_frames) + 1
    h_pos = torch.empty((F, n, 2), dtype=dtype, device=dev)
    h_rot = torch.empty((F, n), dtype=dtype, device=dev)
    h_bond = torch.empty((F, len(bonds)), dtype=torch.bool, device=dev)
    h_sub = torch.empty((F, n), dtype=dtype, device=dev)
    h_eta = torch.empty((max(int(n_frames), 1), 3), dtype=dtype, device=dev)
    h_F = torch.empty((max(int(n_frames), 1), 2), dtype=dtype, device=dev)
    h_J = torch.empty((max(int(n_frames), 1),), dtype=dtype, device=dev)
    h_pos[0], h_rot[0], h_bond[0], h_sub[0] = state.positions, state.rotations, state.bond_intact, state.submergence
    kept = 1  # frames stored (including the initial one)
    frames_run = 0  # frames whose impulse counts (goal trimming does not remove them)
    frame_start = 0
    use_ship_dynamics = ship_trajectory is not None
    while frame_start < n_frames:
        frame_end = min(frame_start + chunk, n_frames)
        K = frame_end - frame_start
        if use_ship_dynamics and replan_callback is not None:
            world_polygons = None if skip_polygon_extraction else _world_polygons(state, ctx.static)
            pos_np = state.positions.detach().cpu().numpy()
            eta_np = ship_state.eta.detach().cpu().numpy()
            new_traj = replan_callback(frame_start, world_polygons, pos_np.copy(),
                                       ctx.static.thicknesses.detach().cpu().numpy(), eta_np[:2].copy(),
                                       float(eta_np[2]), n_frames - frame_start)
            if new_traj is not None and len(new_traj) >= 1:
                new_traj = _trajectory_to_arr(new_traj)
                new_traj = new_traj[:len(ship_trajectory) - frame_start]
                end_slice = frame_start + len(new_traj)
                ship_trajectory[frame_start:end_slice] = new_traj
                if end_slice < len(ship_trajectory):
                    ship_trajectory[end_slice:] = new_traj[-1]
        # setpoints of the chunk (jax_simulation.py:1591-1609), padded to the chunk length (:1640-1647)
        frames = np.arange(frame_start, frame_start + chunk)
        frames = np.minimum(frames, frame_end - 1)  # padding repeats the last row
        if ship_trajectory is not None:
            last = len(ship_trajectory) - 1
            sp = np.concatenate([ship_trajectory[np.minimum(frames, last)],
                                 ship_trajectory[np.minimum(frames + 1, last)]], 1)
            sp_t = torch.as_tensor(sp, dtype=dtype, device=dev)
        else:
            eta0 = ship_state.eta.to(dtype)
            sp_t = torch.cat([eta0, eta0]).reshape(1, 6).repeat(chunk, 1)
        # current (jax_simulation.py:1628-1638, the NumPy models' path): every frame of
        # the chunk samples the model at the chunk-start positions, then steps it;
        # padded frames repeat the last row (:1645-1647)
        if ocean_current is None:
            vw = torch.zeros((chunk, n, 2), dtype=dtype, device=dev)
            vws = torch.zeros((chunk, 2), dtype=dtype, device=dev)
        else:
            pos_np = state.positions.detach().cpu().numpy().astype(np.float64)
            ship_xy = ship_state.eta.detach().cpu().numpy()[:2].reshape(1, 2).astype(np.float64)
            v_rows, vs_rows = [], []
            for _ in range(K):
                v_rows.append(np.asarray(ocean_current.sample_batch(pos_np), np.float64))
                vs_rows.append(np.asarray(ocean_current.sample_batch(ship_xy)[0], np.float64))
                ocean_current.step()
            v_rows += [v_rows[-1]] * (chunk - K)
            vs_rows += [vs_rows[-1]] * (chunk - K)
            vw = torch.as_tensor(np.stack(v_rows), dtype=dtype, device=dev)
            vws = torch.as_tensor(np.stack(vs_rows), dtype=dtype, device=dev)
        final_state, final_ship, hist = ctx.scan_segment(state, ship_state, sp_t, vw, vws)
        pos_K, rot_K, bond_K, eta_K, sub_K, j_K, f_K = hist
        h_pos[kept:kept + K] = pos_K[:K]
        h_rot[kept:kept + K] = rot_K[:K]
        h_bond[kept:kept + K] = bond_K[:K]
        h_sub[kept:kept + K] = sub_K[:K]
        h_eta[frame_start:frame_end] = eta_K[:K]
        h_F[frame_start:frame_end] = f_K[:K]
        h_J[frame_start:frame_end] = j_K[:K]
        kept += K
        frames_run = frame_end
        if frame_callback is not None:
            frame_callback(frame_end - 1, pos_K[K - 1].cpu().numpy(), rot_K[K - 1].cpu().numpy(),
                           bond_K[K - 1].cpu().numpy(), eta_K[K - 1, :2].cpu().numpy(), float(eta_K[K - 1, 2]))
        eta_np = eta_K[:K].detach().cpu().numpy()  # the only per-chunk download
        ship_xy = eta_np[-1, :2]
        state, ship_state = final_state, final_ship
        if goal_y_line is not None:
            if ship_xy[1] >= goal_y_line - goal_tolerance:
                crossed = eta_np[:, 1] >= goal_y_line - goal_tolerance
                actual = frame_start + int(np.argmax(crossed)) + 1
                kept = min(kept, actual + 1)
                frame_end = actual
                break
        elif goal_point is not None:
            if np.linalg.norm(ship_xy - np.asarray(goal_point)) <= goal_tolerance:
                break
        if verbose:
            print(f"  [DEM-chunked] frame={frame_end}/{n_frames} ship_y={float(ship_xy[1]):.1f}", flush=True)
        frame_start = frame_end

    n_ship = kept - 1
    eta_h = h_eta[:n_ship].detach().cpu().numpy()
    ship_history = [(eta_h[f, :2].copy(), float(eta_h[f, 2])) for f in range(n_ship)]
    # impulse summed frame by frame in float64, as the reference (:1670)
    j_np = h_J[:frames_run].detach().cpu().numpy().astype(np.float64)
    j_cum = []
    J_cumul = 0.0
    for v in j_np:
        J_cumul += float(v)
        j_cum.append(J_cumul)
    damage_summary = {"impulse_total": J_cumul}
    out = (DeviceHistory(h_pos, kept), DeviceHistory(h_rot, kept), DeviceHistory(h_bond, kept), ship_history,
           DeviceHistory(h_sub, kept))
    if return_ship_diagnostics:
        Fh = h_F[:n_ship].detach().cpu().numpy()
        diags = [{"t": f * dt, "F_ice_ship": Fh[f], "ship_pos": eta_h[f, :2].copy(), "impulse_cumul": j_cum[f]}
                 for f in range(n_ship)]
        if diags:
            diags[-1]["damage_summary"] = damage_summary
        return out + (diags,)
    return out + (damage_summary,)
