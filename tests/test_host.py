"""Host-side logic: static-data and vessel builders vs the reference's builders."""
import numpy as np
import pytest

from helpers import B_THRUST, SMALL_FLEX, default_cfg
from mbd_icenav_b200.config import IceMaterial
from mbd_icenav_b200.state import build_static_arrays, initial_ice_state_arrays, ship_dynamics_arrays
from mbd_icenav_b200.vessel import ShipProperties

STATIC_CMP = ("local_polys_padded", "poly_mask", "poly_n_verts", "masses", "inertia", "radii",
              "areas", "thicknesses", "bond_i", "bond_j", "rest_lengths", "bond_strengths",
              "bond_areas", "sigma_bar_bond", "initial_floe_of")


def _cmp_static(ours, g, prefix):
    for k in STATIC_CMP:
        a = np.asarray(getattr(ours, k))
        b = np.asarray(g[f"{prefix}_static_{k}"])
        assert a.shape == b.shape, k
        if a.dtype.kind in "biu":
            np.testing.assert_array_equal(a, b, err_msg=k)
        else:
            np.testing.assert_allclose(a, b, rtol=1e-14, atol=1e-300, err_msg=k)
    assert abs(ours.k_n - float(g[f"{prefix}_static_k_n"])) <= 1e-6 * ours.k_n
    assert abs(ours.k_s - float(g[f"{prefix}_static_k_s"])) <= 1e-6 * ours.k_s


def test_static_builder_random_polys(golden64):
    g = golden64
    n = int(g["fn_npoly"])
    polys = [g[f"fn_poly_{i}"] for i in range(n)]
    bonds = [tuple(b) for b in g["fn_bonds"].tolist()]
    ours = build_static_arrays(polys, g["fn_pos"], bonds, g["fn_thick"], g["fn_parents"], default_cfg())
    _cmp_static(ours, g, "fn")


def test_static_builder_small_field(golden64):
    from mbd_icenav_b200 import scene
    f = scene.make_small_field(seed=0, n_frames=300)
    np.testing.assert_array_equal(f.centroids, golden64["small_centroids"])
    mat = IceMaterial(ice_density=900.0, flexural_strength_base=SMALL_FLEX)
    ours = build_static_arrays(f.polygons, f.centroids, f.bonds, f.thicknesses, f.parent_ids,
                               default_cfg(), material=mat, dilation=0.05)
    _cmp_static(ours, golden64, "small")


def test_ship_dynamics_builder(golden64):
    g = golden64
    ours = ship_dynamics_arrays(ShipProperties(length=40.0, beam=8.0, draft=3.0), default_cfg(), 40.0, 8.0)
    for k in ("M3inv", "D3", "Kp", "Kd", "Ki", "B_pinv", "n_max", "ship_hull_local"):
        np.testing.assert_allclose(getattr(ours, k), g[f"fn_shipdyn_{k}"], rtol=1e-12, atol=1e-12, err_msg=k)
    assert ours.mass == pytest.approx(float(g["fn_shipdyn_mass"]), rel=1e-15)
    assert ours.Izz == pytest.approx(float(g["fn_shipdyn_Izz"]), rel=1e-15)


def test_initial_state_layout():
    st = initial_ice_state_arrays(5, np.arange(10.0).reshape(5, 2), 3, np.array([0, 0, 1, 2, 2]))
    assert st.positions.shape == (5, 2) and st.bond_intact.dtype == bool and st.bond_intact.all()
    assert st.dpdem_floe_eligible.shape == (3,) and not st.elem_active.any()
    assert st._fields == ("positions", "velocities", "rotations", "angular_vels", "submergence",
                          "bond_intact", "bond_damage", "bond_delta_m_0", "bond_delta_m_max",
                          "bond_delta_s", "elem_active", "dpdem_floe_eligible")


def test_scene_presets_shapes():
    from mbd_icenav_b200 import scene
    f = scene.make_small_field(seed=1)
    assert f.n == 24 and 20 <= len(f.bonds) <= 80
    assert all(len(p) >= 3 for p in f.polygons)
    assert all(i < j for i, j in f.bonds)
    assert f.setpoints(0, 4).shape == (4, 6)
    assert f.hull_local.shape == (7, 2)
