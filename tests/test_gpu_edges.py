"""Edge cases of the frame step on the GPU, against the oracle (float64).

* A field with no bonds at all: the bond paths (slot records, bond stamps,
  fracture) run on empty arrays.
* A state whose elements are all active from the first frame: every element
  moves and integrates, where the other tests start from frozen ice.

Both push a ship through a row of hexagonal elements for 40 frames of 5
substeps, stepped as one scan, and compare positions, velocities, activation,
bond masks and the ship pose with the oracle's frame loop (1e-9 relative).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

K = 40
K_SUB = 5


def _field(n_cells: int, bonded: bool):
    ang = np.linspace(0, 2 * np.pi, 7)[:-1]
    hexp = np.column_stack([2.0 * np.cos(ang), 2.0 * np.sin(ang)])
    cents = np.array([[4.0 * i, 0.3 * (i % 2)] for i in range(n_cells)])
    polys = [hexp + c for c in cents]
    bonds = [(i, i + 1) for i in range(n_cells - 1)] if bonded else []
    parents = np.zeros(n_cells, np.int32) if bonded else np.arange(n_cells, dtype=np.int32)
    return polys, cents, bonds, parents


def _run(polys, cents, bonds, parents, all_active: bool):
    from mbd_icenav_b200 import sim
    from mbd_icenav_b200.config import SimulationConfig
    from mbd_icenav_b200.state import (build_initial_ice_state, build_initial_ship_state, build_ship_dynamics_data,
                                       build_static_arrays, build_static_data, initial_ice_state_arrays,
                                       ship_dynamics_arrays, to_numpy)
    from mbd_icenav_b200.vessel import ShipProperties, SupplyVessel
    from oracle.dem_oracle import OShip, OState, Oracle, params_from_config
    dev = torch.device("cuda", 0)
    n, nb = len(polys), len(bonds)
    cfg = SimulationConfig()
    props = ShipProperties(length=15.0, beam=5.0, draft=2.5)
    sv = SupplyVessel(mass=props.mass, length=15.0)
    dt = 0.05
    static = build_static_data(polys, cents, bonds, np.ones(n), parents, cfg, device=dev, dtype=torch.float64)
    sdyn = build_ship_dynamics_data(props, cfg, 15.0, 5.0, device=dev, dtype=torch.float64)
    fs = sim.make_frame_step(static, cfg, sdyn, 15.0, 5.0, K_SUB, dt, dt / K_SUB, False, sv.B, sv.T_n)
    st = build_initial_ice_state(n, cents, nb, parents, device=dev, dtype=torch.float64)
    if all_active:
        st = st._replace(elem_active=torch.ones(n, dtype=torch.bool, device=dev))
    eta0 = np.array([-9.0, 0.2, 0.0])  # bow (x = -1.5) inside the first element
    ship = build_initial_ship_state(eta0[:2], 0.0, device=dev, dtype=torch.float64)
    path = np.array([[eta0[0] + 0.15 * i, eta0[1], 0.0] for i in range(K + 1)])  # 3 m/s along +x
    rows = torch.as_tensor(np.concatenate([path[:K], path[1:]], 1), dtype=torch.float64, device=dev)
    vw = torch.zeros((K, n, 2), dtype=torch.float64, device=dev)
    fin, fship, hist = fs.scan_segment(st, ship, rows, vw)
    g = to_numpy(fin)
    # the oracle's frame loop
    sa = build_static_arrays(polys, cents, bonds, np.ones(n), parents, cfg)
    oracle = Oracle(sa, ship_dynamics_arrays(props, cfg, 15.0, 5.0),
                    params_from_config(cfg, 15.0, 5.0, K_SUB, dt, dt / K_SUB, False, sv.T_n), sv.B)
    ost = OState(*initial_ice_state_arrays(n, cents, nb, parents))
    if all_active:
        ost = ost._replace(elem_active=np.ones(n, bool))
    osh = OShip(eta0.copy(), np.zeros(3), np.zeros(6), np.zeros(3))
    for f in range(K):
        ost, osh, _ = oracle.frame_step(ost, osh, path[f], path[f + 1], np.zeros((n, 2)), ost.dpdem_floe_eligible)
    scale = max(1.0, float(np.abs(ost.positions).max()))
    assert np.abs(g.positions - ost.positions).max() / scale < 1e-9
    vs = max(1e-3, float(np.abs(ost.velocities).max()))
    assert np.abs(g.velocities - ost.velocities).max() / vs < 1e-9
    np.testing.assert_array_equal(g.elem_active, ost.elem_active)
    np.testing.assert_array_equal(g.bond_intact, ost.bond_intact)
    np.testing.assert_allclose(fship.eta.cpu().numpy(), osh.eta, rtol=1e-9, atol=1e-9)
    fs.close()
    return g, ost


def test_field_without_bonds_follows_the_oracle():
    polys, cents, bonds, parents = _field(6, bonded=False)
    g, ost = _run(polys, cents, bonds, parents, all_active=False)
    assert g.bond_intact.size == 0
    assert g.elem_active.any()                             # the ship met the elements
    assert np.abs(g.positions - cents).max() > 1e-3        # and moved them


def test_all_elements_active_from_the_start_follow_the_oracle():
    polys, cents, bonds, parents = _field(6, bonded=True)
    g, ost = _run(polys, cents, bonds, parents, all_active=True)
    assert g.elem_active.all()
