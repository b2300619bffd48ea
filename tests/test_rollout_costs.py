"""Per-rollout planner costs (``dem_rollout_costs``).

CPU: the oracle's float32 restatement of the planner's raw cost components
equals the reference's ``_make_raw_components_fn`` run under the NumPy jax shim
bit for bit (``tests/golden/rollout_cost_golden.npz``: hull-corner and
centre-only queries, out-of-bounds penalties, goal-line truncation).

GPU: the kernel gives the same four components for the golden paths within
float32 summation-order tolerance (rtol 1e-5): the kernel sums waypoints in
order, the reference's reductions pair them.
"""
import os
from types import SimpleNamespace

import numpy as np
import pytest

from oracle.rollout_oracle import raw_components, transferred_ke, waypoint_costs

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "rollout_cost_golden.npz")
RTOL = 1e-5


def _meta(g):
    m = g["meta"]
    return dict(x_origin=float(m[0]), y_origin=float(m[1]), resolution=float(m[2]), rows=int(m[3]), cols=int(m[4]))


def _trunc(g, q):
    return None if np.isnan(g["trunc"][q]) else float(g["trunc"][q])


def test_oracle_costs_match_reference_bit_for_bit():
    g = np.load(GOLDEN)
    meta = _meta(g)
    for q in range(len(g["traj"])):
        r = raw_components(g["traj"][q], g["u_norm"][q], g["grid"], meta, g["goal"], g["hull"][q, 0],
                           g["hull"][q, 1], _trunc(g, q))
        np.testing.assert_array_equal(r, g["raw"][q], err_msg=f"path {q}")
    # the cases the golden set covers
    assert (g["raw"][:, 0] >= 1e8).any() and (g["raw"][:, 0] < 1e8).any()
    assert np.isnan(g["trunc"]).any() and (~np.isnan(g["trunc"])).any()
    assert (g["hull"][:, 0] == 0).any() and (g["hull"][:, 0] > 0).any()


def test_transferred_ke_oracle():
    m = np.array([1.0, 2.0, 3.0, 4.0])
    v0 = np.zeros((4, 2))
    v1 = np.array([[1.0, 0.0], [0.0, 1.0], [1.0, 1.0], [0.0, 0.0]])
    np.testing.assert_allclose(transferred_ke(m, v0, v1, [0, 1, 4]), [0.5, 1.0 + 3.0])


@pytest.mark.gpu
def test_gpu_costs_match_reference():
    torch = pytest.importorskip("torch")
    from mbd_icenav_b200 import rollouts
    g = np.load(GOLDEN)
    meta = _meta(g)
    d = torch.device("cuda", 0)
    cm = SimpleNamespace(grid=torch.as_tensor(g["grid"], device=d), **meta)
    center = g["center"].astype(np.float32)
    scale = g["scale"].astype(np.float32)
    for q in range(len(g["traj"])):
        tr = torch.as_tensor(g["traj"][q], device=d)                       # (H+1, 3) float32
        u = g["u_norm"][q] * scale + center                                   # the planner's u_phys (float32)
        out = rollouts.path_costs(tr[0:1], tr[1:, None, :], torch.as_tensor(u[:, None, :], device=d), cm, g["goal"],
                                  float(g["hull"][q, 0]), float(g["hull"][q, 1]), center, scale,
                                  cost_truncate_y=_trunc(g, q)).cpu().numpy()
        np.testing.assert_allclose(out[0, :4], g["raw"][q], rtol=RTOL, atol=1e-6, err_msg=f"path {q}")
        assert out[0, 4] == 0.0  # no masses given: no kinetic energy term


@pytest.mark.gpu
def test_gpu_waypoint_costs_match_oracle():
    """dem_rollout_waypoint_costs: the per-pose costmap value inside the cost
    term, for every golden path's poses after step 0, hull and centre-only;
    within 1e-5 relative (the device's float32 sine and cosine may differ from
    NumPy's by an ulp, which moves a corner query by as much)."""
    torch = pytest.importorskip("torch")
    from mbd_icenav_b200 import rollouts
    g = np.load(GOLDEN)
    meta = _meta(g)
    d = torch.device("cuda", 0)
    cm = SimpleNamespace(grid=torch.as_tensor(g["grid"], device=d), **meta)
    for q in range(len(g["traj"])):
        L, B = float(g["hull"][q, 0]), float(g["hull"][q, 1])
        tr = torch.as_tensor(g["traj"][q], device=d)
        got = rollouts.waypoint_costs(tr[1:, None, :], cm, L, B).cpu().numpy()[0]
        want = waypoint_costs(g["traj"][q][1:], g["grid"], meta, L, B)
        np.testing.assert_allclose(got, want, rtol=RTOL, atol=1e-6, err_msg=f"path {q}")
    # several paths at once, laid out (H, Q, 3): row q of the output is path q
    Hm = min(len(t) for t in g["traj"]) - 1
    stack = np.stack([t[1:Hm + 1] for t in g["traj"]], 1)
    got = rollouts.waypoint_costs(torch.as_tensor(stack, device=d), cm, 60.0, 12.0).cpu().numpy()
    for q in range(stack.shape[1]):
        np.testing.assert_allclose(got[q], waypoint_costs(stack[:, q], g["grid"], meta, 60.0, 12.0), rtol=RTOL,
                                   atol=1e-6, err_msg=f"stacked path {q}")
