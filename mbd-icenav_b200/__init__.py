"""B200-native DPDEM ice-ship frame step (drop-in for ``medea_ice_ship.jax_simulation``).

The directory name contains a hyphen, so it is imported under the alias
``mbd_icenav_b200`` (see ``load_package`` in ``_pkg.py`` beside this file).
"""
from .config import IceMaterial, SimulationConfig, get_default_simulation_config  # noqa: F401
from .state import (IceState, IceStaticData, ShipDynamicsData, ShipState,  # noqa: F401
                    build_initial_ice_state, build_initial_ship_state,
                    build_ship_dynamics_data, build_static_data)
