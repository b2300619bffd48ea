"""Configuration objects read by the DEM frame step.

``SimulationConfig`` carries the same field names and defaults as the
reference's ``medea_ice_ship/config.py:46-227`` for every field the hot path
reads (``jax_simulation.py:325-361``), so a reference config object can be
passed in its place (fields are read by name with ``getattr``).

``IceMaterial`` holds the constants the reference keeps as class attributes of
``IceProperties`` (``medea_ice_ship/properties.py:6-22``).  They are explicit
here so a run can change them (the small three-floe workload uses a 900 kg/m^3
ice density and a 0.5 MPa strength) without patching a class.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional, Tuple

import numpy as np


@dataclass(frozen=True)
class IceMaterial:
    """Ice/water constants (``properties.py:6-22``)."""

    ice_density: float = 920.0
    water_density: float = 1025.0
    flexural_strength_base: float = 0.3e6
    youngs_modulus: float = 5e9

    def flexural_strength(self, thickness):
        # properties.py:14-16: sigma_f = base * sqrt(h / 1.0)
        return self.flexural_strength_base * np.sqrt(thickness / 1.0)

    def breaking_force(self, thickness, width):
        # properties.py:18-22: F = sigma_f * w * h^2
        return self.flexural_strength(thickness) * width * thickness ** 2


DEFAULT_MATERIAL = IceMaterial()


@dataclass(frozen=True)
class SimulationConfig:
    """Fields of the reference ``SimulationConfig`` that the frame step uses."""

    dt: float = 0.05
    use_rayleigh_dt_cap: bool = False
    rayleigh_safety_factor: float = 0.1
    pen_crit_ref: float = 0.5
    pen_crit_thickness_ref: float = 1.0
    max_fracture_thickness: float = 15.0
    n_edge_samples: int = 4
    w_contact_radius_factor: float = 2.0
    w_contact_cap: float = 4.0
    side_push_factor: float = 0.2
    submergence_rate: float = 0.4
    submergence_pen_cap: float = 0.5
    rise_time_const: float = 0.5
    max_bond_width: float = 4.0
    bond_stiffness_factor: float = 0.001
    poisson_ratio: float = 0.3
    bond_cohesion: float = 1.8e6
    bond_internal_friction: float = 0.7
    bond_G_c_I: float = 12.0
    bond_G_c_II: float = 12.0
    bond_eta_bk: float = 1.75
    ice_ice_friction: float = 0.1
    hertz_factor: float = 2e5
    hertz_exponent: float = 1.5
    friction_cap: float = 1e5
    c_d_drag: float = 0.4
    drag_ref_thickness: float = 1.0
    linear_drag_factor: float = 0.1
    drag_coefficient_moment: float = 0.4
    velocity_clip: Tuple[float, float] = (-20.0, 20.0)
    stress_transfer: float = 0.3
    stress_diffusion_steps: int = 2
    effective_strength_collision: float = 0.1
    angular_damping: float = 0.85
    angular_cap: Tuple[float, float] = (-0.2, 0.2)
    ship_velocity_clip: Tuple[float, float, float] = (15.0, 8.0, 0.15)
    max_ship_ice_force: Optional[float] = 25e6
    ice_brake_threshold: float = 0.0
    position_clip_m: float = 1e4


def get_default_simulation_config() -> SimulationConfig:
    return SimulationConfig()


# Defaults the reference's frame-step factory applies with getattr when a
# config object lacks the field (jax_simulation.py:327, :337, :343, :354, :356).
_FACTORY_DEFAULTS = {"n_edge_samples": 3, "drag_coefficient_moment": 0.4,
                     "position_clip_m": 1e4, "max_fracture_thickness": 15.0,
                     "ice_brake_threshold": 0.0, "poisson_ratio": 0.3}


def cfg_get(cfg, name):
    """Read a config field by name, with the reference's fallback defaults."""
    if hasattr(cfg, name):
        return getattr(cfg, name)
    if name in _FACTORY_DEFAULTS:
        return _FACTORY_DEFAULTS[name]
    return getattr(SimulationConfig(), name)
