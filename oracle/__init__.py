"""CPU oracle for the DPDEM ice-ship frame step.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline / reference legs of ``bench.py`` import this package, and only as
the checker or the timed CPU baseline.  The product path (``mbd-icenav_b200``)
never imports it and has no CPU fallback.

``dem_oracle`` restates, in NumPy, the reference's frame step
(``medea_ice_ship/jax_simulation.py:302-701``) and the functions it calls
(``jax_geometry.py``, ``jax_bond_fracture.py``, ``jax_vessel_dynamics.py``).
Parity is pinned: the restatement is checked against golden vectors made by
running the reference's own ``jax_*.py`` files under a NumPy ``jax`` shim
(``tests/golden/make_golden.py``), in float64 and float32.
"""
