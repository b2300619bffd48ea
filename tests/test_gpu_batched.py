"""Several independent systems (ice window + ship) in one handle, on the GPU.

Three copies of the 500-element window occupy the same space; the middle
system's ship starts 5 m to the side.  Stepped together through one
dem_scan_segment launch, every system must reproduce, bit for bit, the
single-system run with its own ship: no contact, bond or force crosses a
system boundary, and each system's force sums are grouped as when it runs
alone.
"""
from types import SimpleNamespace

import numpy as np
import pytest

from helpers import (B_THRUST, SCENARIOS, default_cfg, frame_inputs, gpu_frame_step, initial_state,
                     shipdyn_from_golden, static_from_golden, to_gpu_state)

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

Q = 3
K = 3


def _batched_static(st, q):
    n = st.masses.shape[0]
    nf = int(st.initial_floe_of.max()) + 1
    tile = lambda a: np.concatenate([np.asarray(a)] * q, 0)
    d = {k: tile(getattr(st, k)) for k in ("local_polys_padded", "poly_mask", "poly_n_verts", "masses", "inertia",
                                           "radii", "areas", "thicknesses", "rest_lengths", "bond_strengths",
                                           "bond_areas", "sigma_bar_bond")}
    d["bond_i"] = np.concatenate([np.asarray(st.bond_i) + i * n for i in range(q)])
    d["bond_j"] = np.concatenate([np.asarray(st.bond_j) + i * n for i in range(q)])
    d["initial_floe_of"] = np.concatenate([np.asarray(st.initial_floe_of) + i * nf for i in range(q)])
    d["k_n"], d["k_s"] = st.k_n, st.k_s
    d["pair_i"] = d["pair_j"] = None
    return SimpleNamespace(**d), n


def _inputs(g, prefix, dtype, q):
    d = torch.device("cuda", 0)
    t = lambda a: torch.as_tensor(np.asarray(a, np.float64)).to(d, dtype)
    rows = np.stack([np.concatenate(frame_inputs(g, prefix, f)[:2]) for f in range(K)])
    vw = np.stack([frame_inputs(g, prefix, f)[2] for f in range(K)])
    vws = np.stack([frame_inputs(g, prefix, f)[3] for f in range(K)])
    if q == 1:
        return t(rows), t(vw), t(vws)
    return (t(np.repeat(rows[:, None], q, 1)), t(np.concatenate([vw] * q, 1)), t(np.repeat(vws[:, None], q, 1)))


def test_systems_in_one_launch_match_single_runs(golden64):
    from mbd_icenav_b200 import sim
    from mbd_icenav_b200.config import IceMaterial
    g = golden64
    prefix = "window"
    dt = torch.float64
    L, B, k, dt_f, dti, auto, flex = SCENARIOS[prefix]
    st1 = static_from_golden(g, prefix)
    stq, n = _batched_static(st1, Q)
    fsq = sim.make_frame_step(stq, default_cfg(), shipdyn_from_golden(g, prefix), L, B, k, dt_f, dti, auto,
                              B_THRUST, 1.0, material=IceMaterial(flexural_strength_base=flex),
                              device=torch.device("cuda", 0), dtype=dt, system_start=[i * n for i in range(Q + 1)])
    o_st, o_sh = initial_state(g, prefix, np.float64)
    etas = [o_sh.eta.copy() for _ in range(Q)]
    etas[1] = etas[1] + np.array([5.0, 0.0, 0.0])
    # the batched run
    tile = lambda a: np.concatenate([np.asarray(a)] * Q, 0)
    bst = o_st._replace(**{f: tile(getattr(o_st, f)) for f in o_st._fields})
    bsh = o_sh._replace(eta=np.stack(etas), nu=np.tile(o_sh.nu, (Q, 1)), n_actual=np.tile(o_sh.n_actual, (Q, 1)),
                        e_int=np.tile(o_sh.e_int, (Q, 1)))
    qst, qsh = to_gpu_state(bst, bsh, dt)
    q_fin, q_ship, q_hist = fsq.scan_segment(qst, qsh, *_inputs(g, prefix, dt, Q))
    nb = int(np.asarray(st1.bond_i).shape[0])
    nf = int(np.asarray(st1.initial_floe_of).max()) + 1
    for i in range(Q):
        fs1 = gpu_frame_step(g, prefix, dt)
        sst, ssh = to_gpu_state(o_st, o_sh._replace(eta=etas[i]), dt)
        s_fin, s_ship, s_hist = fs1.scan_segment(sst, ssh, *_inputs(g, prefix, dt, 1))
        el, bo, fl = slice(i * n, (i + 1) * n), slice(i * nb, (i + 1) * nb), slice(i * nf, (i + 1) * nf)
        for name, a, b in zip(s_fin._fields, q_fin, s_fin):
            part = {"bond_intact": bo, "bond_damage": bo, "bond_delta_m_0": bo, "bond_delta_m_max": bo,
                    "bond_delta_s": bo, "dpdem_floe_eligible": fl}.get(name, el)
            assert torch.equal(a[part], b), (i, name)
        for name, a, b in zip(s_ship._fields, q_ship, s_ship):
            assert torch.equal(a[i], b), (i, name)
        assert torch.equal(q_hist[0][:, el], s_hist[0])
        assert torch.equal(q_hist[3][:, i], s_hist[3])  # ship poses
        assert torch.equal(q_hist[6][:, i], s_hist[6])  # forces on the ship
        fs1.close()
    # the shifted ship really made a different run
    assert not torch.equal(q_fin.positions[0:n], q_fin.positions[n:2 * n])
    fsq.close()


def test_single_frame_entry_refuses_several_systems(golden64):
    from mbd_icenav_b200 import _abi, sim
    from mbd_icenav_b200.config import IceMaterial
    g = golden64
    L, B, k, dt_f, dti, auto, flex = SCENARIOS["window"]
    stq, n = _batched_static(static_from_golden(g, "window"), 2)
    fsq = sim.make_frame_step(stq, default_cfg(), shipdyn_from_golden(g, "window"), L, B, k, dt_f, dti, auto,
                              B_THRUST, 1.0, material=IceMaterial(flexural_strength_base=flex),
                              device=torch.device("cuda", 0), dtype=torch.float64, system_start=[0, n, 2 * n])
    o_st, o_sh = initial_state(g, "window", np.float64)
    tile = lambda a: np.concatenate([np.asarray(a)] * 2, 0)
    bst = o_st._replace(**{f: tile(getattr(o_st, f)) for f in o_st._fields})
    bsh = o_sh._replace(**{f: np.tile(getattr(o_sh, f), (2, 1)) for f in o_sh._fields})
    st, sh = to_gpu_state(bst, bsh, torch.float64)
    sp, spn, vw, vws = frame_inputs(g, "window", 0)
    d = torch.device("cuda", 0)
    t = lambda a: torch.as_tensor(np.asarray(a, np.float64)).to(d, torch.float64)
    with pytest.raises(_abi.DemError):
        fsq(st, sh, t(sp), t(spn), t(np.concatenate([vw, vw])), st.dpdem_floe_eligible, t(vws))
    fsq.close()
