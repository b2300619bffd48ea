"""Golden vectors for the control-driven vessel step of planner rollouts.

Usage (in a container where the reference is mounted):

    python tests/golden/make_rollout_golden.py --ref /root/reference

Runs the reference's own ``ship_euler_step_jax`` and ``_clip_velocity_jax``
(``medea_ice_ship/jax_vessel_dynamics.py:54-84``, ``:233-243``) under the NumPy
``jax`` shim in float64 mode, composed as ``ship_step_jax`` composes them
(``:296-348``) with the controller replaced by a given body-frame control:
``tau = u + R(psi)^T tau_ice`` and the current turned to the body frame.  The
vessel matrices are the small workload's (``golden_f64.npz``).  Output:
``rollout_golden.npz`` (committed).
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True)
    args = ap.parse_args()
    import jaxshim
    ref = jaxshim.load_reference(args.ref, x64=True)
    vd = ref.jax_vessel_dynamics
    import jax.numpy as jnp
    g = np.load(os.path.join(HERE, "golden_f64.npz"))
    M3inv, D3 = g["small_shipdyn_M3inv"], g["small_shipdyn_D3"]
    rng = np.random.default_rng(11)
    N = 64
    eta = np.stack([rng.uniform(-50, 50, N), rng.uniform(-50, 50, N), rng.uniform(-3.1, 3.1, N)], 1)
    nu = np.stack([rng.uniform(-3, 3, N), rng.uniform(-1, 1, N), rng.uniform(-0.2, 0.2, N)], 1)
    u = np.stack([rng.normal(0, 6e5, N), np.zeros(N), rng.normal(0, 1.5e8, N)], 1)
    tau_ice = np.stack([rng.normal(0, 5e5, N), rng.normal(0, 5e5, N), rng.normal(0, 1e7, N)], 1)
    vws = np.stack([rng.uniform(-0.3, 0.3, N), rng.uniform(-0.3, 0.3, N)], 1)
    dt, vc = 0.05, (15.0, 8.0, 0.15)
    eta_o, nu_o = [], []
    for i in range(N):
        c, s = np.cos(eta[i, 2]), np.sin(eta[i, 2])
        R = jnp.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])
        nu_c = R.T @ jnp.array([vws[i, 0], vws[i, 1], 0.0])
        tau = jnp.array(u[i]) + R.T @ jnp.array(tau_ice[i])
        e1, n1 = vd.ship_euler_step_jax(jnp.array(eta[i]), jnp.array(nu[i]), tau, jnp.array(M3inv),
                                        jnp.array(D3), dt, nu_c)
        n1 = vd._clip_velocity_jax(n1, *vc)
        eta_o.append(np.asarray(e1))
        nu_o.append(np.asarray(n1))
    np.savez_compressed(os.path.join(HERE, "rollout_golden.npz"), eta=eta, nu=nu, u=u, tau_ice=tau_ice, vws=vws,
                        M3inv=M3inv, D3=D3, dt=dt, vc=np.array(vc), eta_out=np.stack(eta_o), nu_out=np.stack(nu_o))
    print("rollout golden:", N, "cases")


if __name__ == "__main__":
    main()
