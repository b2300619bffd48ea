"""ctypes bindings of ``include/dem_b200.h`` (the library's C ABI).

The structures below mirror the header field by field.  ``load_library``
returns the loaded ``libdem_b200.so`` and raises if it is missing: there is no
fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os

from .build import LIB_PATH

DEM_OK = 0
DEM_ERR_INVALID = 1
DEM_ERR_CUDA = 2
DEM_ERR_CAPACITY = 3
DEM_ERR_TIMEOUT = 4
DEM_ERR_ALIAS = 5
DEM_F32 = 0
DEM_F64 = 1
DEM_LAUNCH_PERSISTENT = 0
DEM_LAUNCH_PHASED = 1
DEM_SPLIT_AUTO, DEM_SPLIT_THREAD, DEM_SPLIT_CTA, DEM_SPLIT_WARP = 0, 1, 1, 2

_ERR_NAMES = {0: "DEM_OK", 1: "DEM_ERR_INVALID", 2: "DEM_ERR_CUDA", 3: "DEM_ERR_CAPACITY",
              4: "DEM_ERR_TIMEOUT", 5: "DEM_ERR_ALIAS"}

_d = C.c_double
_i = C.c_int32
_vp = C.c_void_p
_u8p = C.POINTER(C.c_uint8)


class DemParams(C.Structure):
    _fields_ = [
        ("half_len", _d), ("half_beam", _d),
        ("n_edge_samples", _i), ("n_ice_steps", _i),
        ("dt", _d), ("dt_ice", _d),
        ("bond_stiffness_factor", _d),
        ("hertz_factor", _d), ("hertz_exponent", _d), ("ice_ice_friction", _d), ("friction_cap", _d),
        ("c_d_drag", _d), ("drag_ref_thickness", _d), ("linear_drag_factor", _d),
        ("drag_coefficient_moment", _d),
        ("angular_damping", _d), ("angular_cap_lo", _d), ("angular_cap_hi", _d),
        ("velocity_clip", _d), ("position_clip", _d),
        ("vc_surge", _d), ("vc_sway", _d), ("vc_yaw", _d),
        ("pen_crit_ref", _d), ("pen_crit_thickness_ref", _d),
        ("w_contact_cap", _d), ("w_contact_radius_factor", _d), ("side_push_factor", _d),
        ("submergence_rate", _d), ("submergence_pen_cap", _d), ("rise_time_const", _d),
        ("effective_strength_collision", _d), ("max_fracture_thickness", _d),
        ("has_max_ship_ice_force", _i), ("use_auto_icenav", _i),
        ("max_ship_ice_force", _d), ("ice_brake_threshold", _d),
        ("bond_cohesion", _d), ("bond_internal_friction", _d), ("bond_G_c_I", _d),
        ("bond_G_c_II", _d), ("bond_eta_bk", _d),
        ("youngs_modulus", _d), ("water_density", _d), ("flexural_strength_base", _d),
        ("T_n", _d),
        ("B_mat", _d * 18),
        ("M3inv", _d * 9), ("D3", _d * 9), ("Kp", _d * 9), ("Kd", _d * 9), ("Ki", _d * 9),
        ("B_pinv", _d * 18), ("n_max", _d * 6),
        ("skin", _d), ("max_neighbors", _i), ("bucket_capacity", _i),
    ]


class DemStatic(C.Structure):
    _fields_ = [
        ("n", _i), ("max_v", _i), ("n_bonds", _i), ("n_floes", _i), ("n_hull", _i),
        ("local_polys_padded", _vp), ("poly_mask", _vp), ("poly_n_verts", _vp),
        ("masses", _vp), ("inertia", _vp), ("radii", _vp), ("areas", _vp), ("thicknesses", _vp),
        ("bond_i", _vp), ("bond_j", _vp), ("rest_lengths", _vp), ("bond_strengths", _vp),
        ("sigma_bar_bond", _vp), ("initial_floe_of", _vp),
        ("k_n", _d), ("k_s", _d),
        ("ship_hull_local", _vp),
        ("n_systems", _i), ("system_start", C.POINTER(_i)),
    ]


class DemIceState(C.Structure):
    _fields_ = [(name, _vp) for name in (
        "positions", "velocities", "rotations", "angular_vels", "submergence", "bond_intact",
        "bond_damage", "bond_delta_m_0", "bond_delta_m_max", "bond_delta_s", "elem_active",
        "dpdem_floe_eligible")]


class DemShipState(C.Structure):
    _fields_ = [("eta", _vp), ("nu", _vp), ("n_actual", _vp), ("e_int", _vp)]


class DemDiag(C.Structure):
    _fields_ = [("pen_max", _vp), ("force_mag", _vp), ("F_ice_on_ship", _vp), ("J_cumul_incr", _vp)]


class DemHistory(C.Structure):
    _fields_ = [("positions", _vp), ("rotations", _vp), ("bond_intact", _vp), ("eta", _vp),
                ("submergence", _vp), ("J_cumul_incr", _vp), ("F_ice_on_ship", _vp)]


class DemInfo(C.Structure):
    _fields_ = [("grid_blocks", _i), ("threads_per_block", _i), ("neighbor_rebuilds", C.c_int64),
                ("max_neighbor_count", _i), ("max_bucket_count", _i), ("hash_buckets", _i),
                ("cell_size", _d), ("escaped_total", C.c_int64), ("rebuilt_lists_total", C.c_int64),
                ("capacity_flags", _i)]


class DemCostmapParams(C.Structure):
    _fields_ = [("x_origin", _d), ("y_origin", _d), ("resolution", _d), ("rows", _i), ("cols", _i),
                ("base_cost", _d), ("collision_cost", _d), ("obs_cost_buffer_factor", _d),
                ("ship_speed", _d), ("ship_mass", _d), ("ke_cost_scale", _d),
                ("dilate_half", _i), ("has_masses", _i), ("ice_resistance_weight", _d), ("sic_scratch", _vp)]


class DemRolloutCostParams(C.Structure):
    _fields_ = [("x_origin", _d), ("y_origin", _d), ("resolution", _d), ("rows", _i), ("cols", _i),
                ("oob_penalty", _d), ("ship_length", _d), ("ship_beam", _d), ("goal_x", _d), ("goal_y", _d),
                ("action_center", _d * 3), ("action_scale", _d * 3), ("has_truncate", _i), ("reserved", _i),
                ("truncate_y", _d)]


EXPORTS = ("dem_create", "dem_frame_step", "dem_scan_segment", "dem_sync_status",
           "dem_set_capacity", "dem_set_launch_mode", "dem_set_work_split", "dem_get_info", "dem_set_profiling",
           "dem_get_phase_times", "dem_get_error", "dem_destroy", "dem_version", "dem_debug_fail_barrier", "dem_ke_costmap", "dem_rollout_segment",
           "dem_rollout_costs", "dem_debug_record_contacts", "dem_rollout_ice_terms", "dem_ship_rollout",
           "dem_rollout_waypoint_costs", "dem_rollout_sweep_features")

_LIB = None


def load_library(path: str = None):
    """Load libdem_b200.so (built by ``build.build_library``); raise if absent.

    ``DEM_B200_LIB`` may name another build of the same library (for tuning runs).
    """
    global _LIB
    if _LIB is not None:
        return _LIB
    path = path or os.environ.get("DEM_B200_LIB") or LIB_PATH
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python mbd-icenav_b200/build.py` "
                          "(there is no CPU fallback for the DEM frame step)")
    lib = C.CDLL(path)
    H = C.c_void_p
    lib.dem_create.argtypes = [C.POINTER(DemParams), C.POINTER(DemStatic), _i, _i, C.POINTER(H)]
    lib.dem_frame_step.argtypes = [H, C.POINTER(DemIceState), C.POINTER(DemIceState),
                                   C.POINTER(DemShipState), C.POINTER(DemShipState),
                                   _vp, _vp, _vp, _vp, _vp, C.POINTER(DemDiag), _vp]
    lib.dem_scan_segment.argtypes = [H, C.POINTER(DemIceState), C.POINTER(DemIceState),
                                     C.POINTER(DemShipState), C.POINTER(DemShipState), _i,
                                     _vp, _vp, _vp, C.POINTER(DemHistory), _vp]
    lib.dem_rollout_segment.argtypes = [H, C.POINTER(DemIceState), C.POINTER(DemIceState),
                                        C.POINTER(DemShipState), C.POINTER(DemShipState), _i,
                                        _vp, _vp, _vp, C.POINTER(DemHistory), _vp]
    lib.dem_sync_status.argtypes = [H, _vp]
    lib.dem_set_capacity.argtypes = [H, _i, _i]
    lib.dem_set_launch_mode.argtypes = [H, _i]
    lib.dem_set_work_split.argtypes = [H, _i, _i]
    lib.dem_get_info.argtypes = [H, C.POINTER(DemInfo)]
    lib.dem_set_profiling.argtypes = [H, _i]
    lib.dem_get_phase_times.argtypes = [H, C.POINTER(C.c_int64), _i, C.POINTER(_i), C.POINTER(C.c_int64)]
    lib.dem_get_error.argtypes = [H, C.c_char_p, C.c_size_t]
    lib.dem_destroy.argtypes = [H]
    lib.dem_debug_fail_barrier.argtypes = [H, _i]
    lib.dem_debug_record_contacts.argtypes = [H, _vp, _i, _vp, _i, _vp]
    lib.dem_rollout_ice_terms.argtypes = [_i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp]
    lib.dem_ship_rollout.argtypes = [C.POINTER(DemParams), _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp]
    lib.dem_ke_costmap.argtypes = [_i, _i, _vp, _vp, _vp, _vp, C.POINTER(DemCostmapParams), _vp, _vp, _vp, _vp]
    lib.dem_rollout_costs.argtypes = [_i, _i, _i, _vp, _vp, _vp, _vp, _vp, C.POINTER(DemRolloutCostParams), _vp,
                                      _vp, _vp, _vp, _vp]
    lib.dem_rollout_waypoint_costs.argtypes = [_i, _i, _i, _vp, _vp, C.POINTER(DemRolloutCostParams), _vp, _vp]
    lib.dem_rollout_sweep_features.argtypes = [_i, _i, _i, _vp, _vp, _i, _vp, _vp, _vp, _i, _vp, _vp, _d, _d, _d,
                                               _vp, _vp]
    lib.dem_version.restype = C.c_char_p
    _bind_surrogate(lib)
    for name in EXPORTS:
        if name != "dem_version":
            getattr(lib, name).restype = C.c_int
    _LIB = lib
    return lib


# surrogate kernels (include/surrogate_b200.h)
SG_OK, SG_ERR_INVALID, SG_ERR_CUDA = 0, 1, 2
SG_OUT_F32, SG_OUT_BF16 = 0, 1
SG_EXPORTS = ("sg_gemm", "sg_im2col", "sg_col2im", "sg_transpose", "sg_colsum", "sg_adam", "sg_mse",
              "sg_pack_rows", "sg_unpack_grad", "sg_to_bf16", "sg_gather_rows")


def _bind_surrogate(lib):
    f = C.c_float
    lib.sg_gemm.argtypes = [_i, _i, _i, _vp, _i, _vp, _i, _vp, _i, _i, _vp, _i, _vp, _i, _vp, _vp]
    lib.sg_im2col.argtypes = [_i, _i, _i, _i, _vp, _i, _vp, _vp]
    lib.sg_col2im.argtypes = [_i, _i, _i, _i, _vp, _i, _vp, _vp, _vp]
    lib.sg_transpose.argtypes = [_i, _i, _vp, _i, _vp, _i, _vp]
    lib.sg_colsum.argtypes = [_i, _i, _vp, _i, _i, _vp, _vp]
    lib.sg_adam.argtypes = [_i, _i, _vp, _vp, _vp, _vp, f, f, f, f, _i, _vp, _i, _vp, _i, _vp]
    lib.sg_mse.argtypes = [_i, _i, _vp, _i, _vp, _i, _vp, _i, _vp, _vp]
    lib.sg_pack_rows.argtypes = [_i, _i, _vp, _i, _vp, _i, _vp, _i, _vp, _i, _vp]
    lib.sg_unpack_grad.argtypes = [_i, _i, _vp, _i, _vp, _vp, _vp]
    lib.sg_to_bf16.argtypes = [C.c_int64, _vp, _vp, _vp]
    lib.sg_gather_rows.argtypes = [_i, C.c_int64, _vp, C.c_int64, _vp, _vp, C.c_int64, _vp]
    for name in SG_EXPORTS:
        getattr(lib, name).restype = C.c_int


class DemError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_ERR_NAMES.get(code, code)}: {msg}")
        self.code = code
