/*
 * dem_b200.h — C ABI of the B200-native DPDEM ice–ship frame step.
 *
 * Drop-in boundary for the reference's per-frame physics,
 * medea_ice_ship/jax_simulation.py:
 *   - dem_create        replaces the factory _make_frame_step(static, cfg, ship_dyn,
 *                       ship_length, ship_beam, n_ice_steps, dt, dt_ice,
 *                       use_auto_icenav, B_mat, T_n)           (jax_simulation.py:302-361)
 *   - dem_frame_step    replaces the returned frame_step(state, ship_state, setpoint,
 *                       setpoint_next, v_water, dpdem_eligible, v_water_ship)
 *                                                              (jax_simulation.py:397-699)
 *   - dem_scan_segment  replaces JaxSimContext.scan_segment(state, ship_state,
 *                       setpoints_K6, v_water_Kn2, v_water_ship_K2)
 *                                                              (jax_simulation.py:1308-1335)
 *   - dem_destroy / dem_get_error / dem_sync_status have no reference counterpart
 *     (XLA owns its buffers; JAX raises Python exceptions).
 *
 * Array conventions (all arrays are DEVICE pointers owned by the caller):
 *   - layouts are those of IceState / ShipState / IceStaticData
 *     (medea_ice_ship/jax_ice_state.py:31-96): (n,2) arrays are row-major interleaved
 *     xy, booleans are one byte (0/1), indices are int32;
 *   - every floating-point array has the handle's dtype (DEM_F32 or DEM_F64);
 *   - the library owns only its scratch (broad-phase grid, neighbour lists, bond CSR,
 *     per-frame reductions, barrier words and the device status word).
 *
 * Semantics: functional like the reference — inputs are never modified, outputs
 * are written to caller buffers.  Output element-kinematics buffers
 * (positions, velocities, rotations, angular_vels) must not alias the inputs
 * (DEM_ERR_ALIAS); every other output may alias its input.
 *
 * Errors: every call returns a status.  Launch/argument errors are returned
 * directly.  Conditions found on the device (neighbour capacity exceeded, a grid
 * barrier that waited past its limit) are written to a device status word that
 * dem_sync_status reads; the step's inputs are untouched, so the caller may grow
 * capacities (dem_set_capacity) and re-run the same call.  Kernels never trap.
 *
 * Threading: a handle is bound to one device and is not thread-safe.  Calls that
 * overlap on the GPU (two streams) race on the handle's scratch.
 */
#ifndef DEM_B200_H
#define DEM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DEM_OK 0
#define DEM_ERR_INVALID 1   /* bad argument, shape or null pointer          */
#define DEM_ERR_CUDA 2      /* a CUDA runtime call failed                    */
#define DEM_ERR_CAPACITY 3  /* neighbour / grid-bucket capacity exceeded     */
#define DEM_ERR_TIMEOUT 4   /* a grid barrier wait exceeded its time limit   */
#define DEM_ERR_ALIAS 5     /* an element-kinematics output aliases an input */

#define DEM_F32 0
#define DEM_F64 1

#define DEM_LAUNCH_PERSISTENT 0  /* one cooperative launch per call, device-side grid barriers */
#define DEM_LAUNCH_PHASED 1      /* one launch per phase (neighbour list rebuilt every substep) */

typedef struct DemHandle DemHandle;

/* Scalar constants of the frame step: the closure constants of _make_frame_step
 * (jax_simulation.py:325-361), the IceProperties constants it reads
 * (properties.py:6-12) and the ShipDynamicsData matrices (jax_ice_state.py:99-116). */
typedef struct DemParams {
    double half_len, half_beam;             /* analytic hull half-length / half-beam [m]   */
    int32_t n_edge_samples;                 /* samples per polygon edge (cfg default 4)      */
    int32_t n_ice_steps;                    /* substeps per frame                            */
    double dt, dt_ice;                      /* frame and substep time steps [s]              */
    double bond_stiffness_factor;
    double hertz_factor, hertz_exponent, ice_ice_friction, friction_cap;
    double c_d_drag, drag_ref_thickness, linear_drag_factor, drag_coefficient_moment;
    double angular_damping, angular_cap_lo, angular_cap_hi;
    double velocity_clip, position_clip;
    double vc_surge, vc_sway, vc_yaw;       /* ship velocity clip                            */
    double pen_crit_ref, pen_crit_thickness_ref;
    double w_contact_cap, w_contact_radius_factor, side_push_factor;
    double submergence_rate, submergence_pen_cap, rise_time_const;
    double effective_strength_collision, max_fracture_thickness;
    int32_t has_max_ship_ice_force;         /* 0: cfg.max_ship_ice_force is None             */
    int32_t use_auto_icenav;
    double max_ship_ice_force;
    double ice_brake_threshold;
    double bond_cohesion, bond_internal_friction, bond_G_c_I, bond_G_c_II, bond_eta_bk;
    double youngs_modulus, water_density, flexural_strength_base;
    double T_n;
    double B_mat[18];                       /* (3,6) thruster configuration, row-major       */
    double M3inv[9], D3[9], Kp[9], Kd[9], Ki[9];
    double B_pinv[18];                      /* (6,3) row-major                               */
    double n_max[6];
    /* broad phase (no reference counterpart: the reference evaluates all pairs) */
    double skin;                            /* Verlet skin [m]; 0 = rebuild every substep    */
    int32_t max_neighbors;                  /* neighbour-list capacity per element           */
    int32_t bucket_capacity;                /* elements per grid-hash bucket                 */
} DemParams;

/* IceStaticData (jax_ice_state.py:59-96) as device pointers.  pair_i/pair_j are not
 * taken: the all-pairs contact list is implied and resolved by the broad phase. */
typedef struct DemStatic {
    int32_t n, max_v, n_bonds, n_floes, n_hull;
    const void* local_polys_padded;   /* (n, max_v, 2) */
    const uint8_t* poly_mask;         /* (n, max_v)    */
    const int32_t* poly_n_verts;      /* (n,)          */
    const void* masses;
    const void* inertia;
    const void* radii;
    const void* areas;
    const void* thicknesses;
    const int32_t* bond_i;
    const int32_t* bond_j;
    const void* rest_lengths;
    const void* bond_strengths;
    const void* sigma_bar_bond;
    const int32_t* initial_floe_of;   /* (n,) parent floe, 0 <= id < n_floes */
    double k_n, k_s;
    const void* ship_hull_local;      /* (n_hull, 2) ShipDynamicsData.ship_hull_local */
    /* Independent systems (no reference counterpart): n_systems > 1 splits the
     * elements into contiguous ranges [system_start[q], system_start[q+1]), each
     * an ice window with its own ship (same hull), advanced together by
     * dem_scan_segment / dem_rollout_segment.  Floes and bonds stay inside one
     * system; elements of different systems never interact.  system_start is a
     * HOST array of n_systems + 1 offsets from 0 to n.  0 or 1: one system. */
    int32_t n_systems;
    const int32_t* system_start;
} DemStatic;

/* IceState (jax_ice_state.py:31-44). */
typedef struct DemIceState {
    void* positions;            /* (n,2) */
    void* velocities;           /* (n,2) */
    void* rotations;            /* (n,)  */
    void* angular_vels;         /* (n,)  */
    void* submergence;          /* (n,)  */
    uint8_t* bond_intact;       /* (n_bonds,) */
    void* bond_damage;
    void* bond_delta_m_0;
    void* bond_delta_m_max;
    void* bond_delta_s;
    uint8_t* elem_active;       /* (n,) */
    uint8_t* dpdem_floe_eligible; /* (n_floes,) */
} DemIceState;

/* ShipState (jax_ice_state.py:47-52). */
typedef struct DemShipState {
    void* eta;       /* (3,) */
    void* nu;        /* (3,) */
    void* n_actual;  /* (6,) */
    void* e_int;     /* (3,) */
} DemShipState;

/* frame_step's diag dict (jax_simulation.py:692-697); any field may be NULL. */
typedef struct DemDiag {
    void* pen_max;        /* (n,) */
    void* force_mag;      /* (n,) */
    void* F_ice_on_ship;  /* (2,) */
    void* J_cumul_incr;   /* ()   */
} DemDiag;

/* scan_segment's stacked history tuple (jax_simulation.py:1316-1324); any field may be NULL. */
typedef struct DemHistory {
    void* positions;       /* (K,n,2)      */
    void* rotations;       /* (K,n)        */
    uint8_t* bond_intact;  /* (K,n_bonds)  */
    void* eta;             /* (K,3)        */
    void* submergence;     /* (K,n)        */
    void* J_cumul_incr;    /* (K,)         */
    void* F_ice_on_ship;   /* (K,2)        */
} DemHistory;

/* Counters for tuning and tests. */
typedef struct DemInfo {
    int32_t grid_blocks;        /* cooperative grid size of the persistent kernel  */
    int32_t threads_per_block;
    int64_t neighbor_rebuilds;  /* neighbour-list builds since create               */
    int32_t max_neighbor_count; /* largest list seen since create                   */
    int32_t max_bucket_count;   /* fullest grid bucket seen since create            */
    int32_t hash_buckets;
    double cell_size;
    int64_t escaped_total;       /* elements re-referenced since create             */
    int64_t rebuilt_lists_total; /* neighbour lists rebuilt since create            */
    int32_t capacity_flags;      /* last DEM_ERR_CAPACITY: 1 grid bucket, 2 neighbour list, 3 both */
} DemInfo;

/* Replaces _make_frame_step (jax_simulation.py:302-361): binds static data and
 * constants, builds the per-element bond lists and allocates scratch on `device`. */
int dem_create(const DemParams* params, const DemStatic* static_data, int dtype, int device,
               DemHandle** out);

/* Replaces frame_step (jax_simulation.py:397-699).  setpoint / setpoint_next (3,),
 * v_water (n,2), dpdem_eligible (n_floes,) and v_water_ship (2,) are device arrays;
 * v_water_ship may be NULL (zero current).  `stream` is a cudaStream_t (NULL = default). */
int dem_frame_step(DemHandle* h, const DemIceState* in, DemIceState* out,
                   const DemShipState* ship_in, DemShipState* ship_out,
                   const void* setpoint, const void* setpoint_next, const void* v_water,
                   const uint8_t* dpdem_eligible, const void* v_water_ship,
                   DemDiag* diag, void* stream);

/* Replaces JaxSimContext.scan_segment (jax_simulation.py:1308-1335): K frames with
 * setpoints (K,6) rows [sp, sp_next], v_water (K,n,2), v_water_ship (K,2) or NULL.
 * Each frame uses the previous frame's dpdem_floe_eligible (jax_simulation.py:1314).
 * With Q = n_systems > 1: ship states are (Q,3) / (Q,6) arrays, setpoints (K,Q,6),
 * v_water_ship (K,Q,2), and the history's eta (K,Q,3), J_cumul_incr (K,Q),
 * F_ice_on_ship (K,Q,2).  hist may be NULL, and so may any of its arrays (that
 * row is then not written). */
int dem_scan_segment(DemHandle* h, const DemIceState* in, DemIceState* out,
                     const DemShipState* ship_in, DemShipState* ship_out, int32_t K,
                     const void* setpoints_K6, const void* v_water_Kn2,
                     const void* v_water_ship_K2, DemHistory* hist, void* stream);

/* Planner rollouts (no single counterpart in the reference, whose planners roll
 * the ship out alone, jax_vessel_dynamics.py:87-122): K frames of the frame step
 * (jax_simulation.py:397-699) in which each system's ship is driven by controls
 * instead of setpoints: tau = u + tau_ice (body frame) through ship_euler_step_jax
 * (jax_vessel_dynamics.py:54-84) and the velocity clip (:233-243), as ship_step_jax
 * (:246-348) with its controller replaced; RPMs and integral error are kept.
 * controls_KQ3 (K, Q, 3) body-frame [X, Y, N] per frame and system (Q = n_systems,
 * 1 for a plain field); v_water (K, n, 2); v_water_ship (K, Q, 2) or NULL; the
 * history is that of dem_scan_segment. */
int dem_rollout_segment(DemHandle* h, const DemIceState* in, DemIceState* out,
                        const DemShipState* ship_in, DemShipState* ship_out, int32_t K,
                        const void* controls_KQ3, const void* v_water_Kn2,
                        const void* v_water_ship_KQ2, DemHistory* hist, void* stream);

/* Synchronise `stream`, return and clear the device status word (DEM_OK if clean). */
int dem_sync_status(DemHandle* h, void* stream);

/* Grow (or shrink) neighbour-list and grid-bucket capacities; reallocates scratch. */
int dem_set_capacity(DemHandle* h, int32_t max_neighbors, int32_t bucket_capacity);

/* DEM_LAUNCH_PERSISTENT (default) or DEM_LAUNCH_PHASED; both give identical results. */
int dem_set_launch_mode(DemHandle* h, int32_t mode);

/* How the work of a substep is split (no reference counterpart; results are
 * identical for every choice, this is for tests and tuning).  force_split:
 * DEM_SPLIT_AUTO (a warp per active element when at most two fall to each warp,
 * else a thread per element), DEM_SPLIT_THREAD or DEM_SPLIT_WARP.  mark_split,
 * for the escape rounds: DEM_SPLIT_AUTO (a CTA per escaped element when they fit
 * one per CTA, else a warp each), DEM_SPLIT_CTA or DEM_SPLIT_WARP.  mark_split
 * also sets the unit of a force phase's list rebuilds and lazy escapes:
 * DEM_SPLIT_AUTO (a CTA each when they are at most a quarter of the CTAs, else
 * a warp each), DEM_SPLIT_CTA (a CTA each up to half the CTAs) or DEM_SPLIT_WARP. */
#define DEM_SPLIT_AUTO 0
#define DEM_SPLIT_THREAD 1
#define DEM_SPLIT_CTA 1
#define DEM_SPLIT_WARP 2
int dem_set_work_split(DemHandle* h, int32_t force_split, int32_t mark_split);

int dem_get_info(DemHandle* h, DemInfo* info);

/* Record, in persistent launches, the device time at which each phase ends
 * (profiling aid; off by default). */
int dem_set_profiling(DemHandle* h, int32_t on);

/* Phase end times of the last persistent call: pairs [phase index, ns] (at most
 * max_pairs), their count, and the launch's start time in ns (globaltimer).
 * Phase indices count 5 + 3 k per frame: cull, near contact, contact forces,
 * reduce, then per substep escape round, all-lists rebuild and force, and
 * fracture.  Phases skipped on the device (no escapes, no full rebuild) record
 * no entry. */
int dem_get_phase_times(DemHandle* h, int64_t* pairs, int32_t max_pairs, int32_t* count, int64_t* start_ns);

/* Failure-detection test hook (no reference counterpart): in the next
 * persistent call on this handle, the last CTA leaves instead of arriving at
 * the grid barrier that follows phase `phase`.  Every other CTA's wait then
 * ends at its time limit (2 s), the call's status becomes DEM_ERR_TIMEOUT and
 * dem_sync_status resets the broad phase, so the handle stays usable.
 * One-shot; DEM_ERR_INVALID in phased mode or for phase < 0. */
int dem_debug_fail_barrier(DemHandle* h, int32_t phase);

/* Contact-set recording, a parity aid (no reference counterpart).  With
 * `pairs` not NULL, every later call on this handle records each ice–ice pair
 * whose contact term a force phase computed — the pairs with overlap > 0 and
 * distance > 1e-6 (jax_simulation.py:127-131) among each active element's
 * candidates — as int32 pairs {e, o} seen from the active element e (a pair
 * of two active elements appears twice, once from each), at most `capacity`
 * pairs; *count (device uint32, zeroed at the start of every call) gets the
 * total, which exceeds capacity if pairs were dropped.  After substep s of
 * frame f of a call, marks[f * n_ice_steps + s] gets the number of pairs
 * recorded so far (for f * n_ice_steps + s < max_marks), so the pairs of one
 * substep are pairs[marks[m-1] .. marks[m]).  Records of one substep come in
 * no fixed order.  All arrays are device arrays owned by the caller;
 * pairs = NULL turns recording off.  Results of the step are unchanged. */
int dem_debug_record_contacts(DemHandle* h, int32_t* pairs, int32_t capacity, int32_t* marks, int32_t max_marks,
                              uint32_t* count);

/* Copy the last error message (NUL-terminated) into buf. */
int dem_get_error(DemHandle* h, char* buf, size_t len);

int dem_destroy(DemHandle* h);

/* Library version string, e.g. "dem_b200 0.1 sm_100a". */
const char* dem_version(void);

/* Grid and cost constants of dem_ke_costmap (arguments of build_costmap_jax,
 * jax_costmap.py:179-203, after its grid geometry, :237-244). */
typedef struct DemCostmapParams {
    double x_origin, y_origin;     /* world position of cell (0,0)'s lower-left corner [m] */
    double resolution;             /* cell size [m]                                      */
    int32_t rows, cols;
    double base_cost;              /* open-water cost                                   */
    double collision_cost;         /* KE cost weight                                    */
    double obs_cost_buffer_factor; /* extra fractional radius painted per element       */
    double ship_speed, ship_mass, ke_cost_scale;
    int32_t dilate_half;           /* square max window of 2h+1 cells; 0 = no dilation  */
    int32_t has_masses;            /* 0: masses = pi r^2 h 920 (jax_costmap.py:257-259) */
    double ice_resistance_weight;  /* > 0: SIC modulation grid * SIC^w (:271-284)       */
    void* sic_scratch;             /* device, rows * cols doubles when the weight is > 0 */
} DemCostmapParams;

/* Replaces the device work of build_costmap_jax (jax_costmap.py:179-331): the KE collision costmap of the ice elements
 * (centroids (n,2), radii, thicknesses, masses (n,) of `dtype`; masses may be
 * NULL when has_masses = 0, thicknesses when it is 1) into grid (rows, cols)
 * float32, row-major, with the SIC modulation when params->ice_resistance_weight
 * > 0.  tmp (rows, cols) float32 is needed when dilate_half > 0; flag is one
 * device int32 of scratch.  All pointers are device pointers; `stream` is a
 * cudaStream_t.  Bit-exact with the reference's float32 grid (for a SIC weight
 * other than 1 the reference's float32 power may differ by one unit in the
 * last place from the device's, which rounds a double power once). */
int dem_ke_costmap(int32_t dtype, int32_t n, const void* centroids, const void* radii,
                   const void* thicknesses, const void* masses, const DemCostmapParams* params,
                   float* grid, float* tmp, int32_t* flag, void* stream);

/* Cost arguments of dem_rollout_costs: the planner's costmap query and cost
 * terms (jax_mbd_planner.py:_make_query :128-168, _make_raw_components_fn
 * :569-665, with the action normalisation of :2782-2783). */
typedef struct DemRolloutCostParams {
    double x_origin, y_origin;     /* costmap geometry (meta of the costmap)            */
    double resolution;
    int32_t rows, cols;
    double oob_penalty;            /* added when a query leaves the grid's x-extent     */
    double ship_length, ship_beam; /* hull centre + 4 box corners when both are > 0     */
    double goal_x, goal_y;
    double action_center[3];       /* u_norm = (u - center) / scale for the jerk term   */
    double action_scale[3];
    int32_t has_truncate;          /* cost_truncate_y given                             */
    int32_t reserved;
    double truncate_y;
} DemRolloutCostParams;

/* Per-rollout costs after dem_rollout_segment (no reference counterpart as a
 * whole; each term follows the reference planner's).  For every system q of
 * n_systems: the pose path eta0[q] (Q,3), eta_hist[:, q] (H,Q,3) (the pose
 * history of the segment) gives out[q] = [costmap integral, path length,
 * discounted goal distance, jerk, transferred kinetic energy] (Q,5) double,
 * the first four in float32 arithmetic as _make_raw_components_fn
 * (jax_mbd_planner.py:569-665) computes its raw components on the costmap
 * grid (rows, cols) float32.  controls (H,Q,3) give the jerk (NULL: 0).
 * masses (n,), vel0 and vel1 (n,2) (the segment's input and output ice
 * velocities) with system_start (Q+1) give sum 0.5 m (|v1|^2 - |v0|^2) over
 * each system's elements in double (all NULL: 0).  All arrays are device
 * arrays of `dtype` (grid float32, system_start int32); 1 <= horizon <= 2000. */
int dem_rollout_costs(int32_t dtype, int32_t n_systems, int32_t horizon, const int32_t* system_start,
                      const void* eta0, const void* eta_hist, const void* controls, const float* grid,
                      const DemRolloutCostParams* params, const void* masses, const void* vel0,
                      const void* vel1, double* out, void* stream);

/* Per-waypoint costmap values of pose paths (the waypoint term inside
 * _make_raw_components_fn, jax_mbd_planner.py:569-665, before the trapezoid
 * rule): out[q, t] (Q, H) float32 = the query (:128-168) at the hull centre
 * and four box corners, maximum (the centre alone when ship_length or
 * ship_beam is 0), of the pose eta_hist[t, q] (H, Q, 3) of `dtype`.  Only the
 * costmap geometry, oob_penalty and the hull size of params are read; grid
 * (rows, cols) float32.  Device arrays; 1 <= horizon <= 2000.  The screening
 * surrogate reads these along each candidate's rigid-ship path. */
int dem_rollout_waypoint_costs(int32_t dtype, int32_t n_systems, int32_t horizon, const void* eta_hist,
                               const float* grid, const DemRolloutCostParams* params, float* out, void* stream);

/* Per-rollout ice terms after dem_rollout_segment (no reference counterpart
 * as a whole): for every system q of n_systems, out[q] (Q,2) double =
 * [hull impulse: the sum over the segment's steps of J_hist[t, q], the
 * frame's |F_ice_on_ship| dt (J_cumul_incr, jax_simulation.py:692-697), in
 * step order; bonds broken: the bonds b in [bond_start[q], bond_start[q+1])
 * with intact0[b] set and intact1[b] clear].  J_hist (H, Q) of `dtype`;
 * bond_start (Q+1) int32 or NULL (no bond count); intact0 / intact1 (n_bonds)
 * the segment's input and output bond_intact.  All device arrays. */
int dem_rollout_ice_terms(int32_t dtype, int32_t n_systems, int32_t horizon, const void* J_hist,
                          const int32_t* bond_start, const uint8_t* intact0, const uint8_t* intact1, double* out,
                          void* stream);

/* The planners' rigid-ship rollout (jax_mbd_planner.py:51-122 rolls the
 * 3-DOF ship out over a static costmap): for each of n_rollouts candidates,
 * `horizon` steps of the vessel update of dem_rollout_segment (tau = u,
 * ship_euler_step_jax and the velocity clip, jax_vessel_dynamics.py:54-84,
 * :233-243) with no ice load.  eta0, nu0 (Q,3); controls (H,Q,3) body-frame
 * [X, Y, N]; v_water_ship (H,Q,2) or NULL; eta_hist (H,Q,3) gets the poses
 * after each step, nu_out (Q,3) (or NULL) the final velocity.  Arrays are
 * device arrays of `dtype`; params supplies dt, D3, M3inv and the clip. */
int dem_ship_rollout(const DemParams* params, int32_t dtype, int32_t n_rollouts, int32_t horizon, const void* eta0,
                     const void* nu0, const void* controls, const void* v_water_ship, void* eta_hist, void* nu_out,
                     void* stream);

/* Features of dem_rollout_sweep_features, and its limits. */
#define DEM_SWEEP_FEATURES 8
#define DEM_SWEEP_MAX_ELEMENTS 65536
#define DEM_SWEEP_MAX_HORIZON 512

/* What each candidate's rigid-ship path sweeps through the plan's ice window
 * (no reference counterpart: inputs of the screening surrogate, beside the
 * path's costmap values).  Poses: eta0[q] (Q,3) and eta_hist[t, q] (H,Q,3)
 * of `dtype`, from dem_ship_rollout.  An element e of the window (positions
 * (n,2), radii, masses (n,) of `dtype`) is hit at the first pose t = 0..H
 * whose frame puts its centroid inside the hull box grown by its radius
 * (|x| < half_len + r, |y| < half_beam + r); the hit's velocity is the path's
 * step velocity (pose t - pose t-1) / dt (the first step's at t = 0) and v_n
 * its component towards the centroid, clamped at 0.  out (Q, 8) float32 =
 * [elements hit, their mass, sum 0.5 m |v|^2, sum m v_n,
 * sum m (H + 1 - t) / (H + 1), sum 0.5 m v_n^2, bonds (bond_i, bond_j (nb)
 * int32 window indices) with one end hit, bonds with both ends hit], summed in
 * double in a fixed order.  Device arrays; n <= DEM_SWEEP_MAX_ELEMENTS,
 * 1 <= horizon <= DEM_SWEEP_MAX_HORIZON. */
int dem_rollout_sweep_features(int32_t dtype, int32_t n_rollouts, int32_t horizon, const void* eta0,
                               const void* eta_hist, int32_t n, const void* positions, const void* radii,
                               const void* masses, int32_t n_bonds, const int32_t* bond_i, const int32_t* bond_j,
                               double half_len, double half_beam, double dt, float* out, void* stream);

/* Largest n accepted by dem_ship_contact_noalloc. */
#define DEM_CONTACT_NOALLOC_MAX_ELEMENTS 262144

/* Ship–ice contact detection that allocates nothing.  No counterpart in the
 * reference: it is the contact test that dem_frame_step runs at the start of
 * every frame (diag.pen_max), offered without a handle for callers that cannot
 * call cudaMalloc — a host whose caching allocator already owns all of the
 * GPU's memory, or a fixed-rate navigation loop that cannot take cudaMalloc's
 * device-wide synchronisation and unbounded latency in its cycle.
 *
 * For each element (positions (n,2), rotations (n,), local_polys_padded
 * (n,max_v,2), poly_mask (n,max_v), all DEVICE arrays of `dtype`) against the
 * ship at ship_eta (3,) with outline ship_hull_local (n_hull,2) and analytic
 * hull half_len x half_beam: pen_max (n,) gets the deepest penetration and, if
 * not NULL, normals (n,2) its unit normal (zeros where there is no contact).
 * Runs on the CURRENT device and on `stream` (a cudaStream_t; NULL = default).
 *
 * Scratch: one static device array of 1 MiB + 256 bytes per device (held by
 * every device that loads the library until the process exits), hence the
 * limit n <= DEM_CONTACT_NOALLOC_MAX_ELEMENTS; larger n returns
 * DEM_ERR_CAPACITY before any work.  Every call made outside stream capture
 * looks up that array's device address on the current device (so a device
 * reset leaves no stale address); a call inside a capture uses the address
 * of the last call outside capture on that device, so make one call before
 * any stream capture on the device, and again after a device reset (a first
 * call inside a capture returns DEM_ERR_INVALID).  Every call on a device shares the array, so
 * calls that overlap on the GPU (other streams, other host threads) race on
 * it: serialise them.  Returns DEM_ERR_INVALID for bad arguments and
 * DEM_ERR_CUDA if a launch fails. */
int dem_ship_contact_noalloc(int32_t dtype, int32_t n, int32_t max_v, const void* local_polys_padded,
                             const uint8_t* poly_mask, const void* positions, const void* rotations,
                             int32_t n_hull, const void* ship_hull_local, double half_len, double half_beam,
                             int32_t n_edge_samples, const void* ship_eta, void* pen_max, void* normals,
                             void* stream);

#ifdef __cplusplus
}
#endif
#endif /* DEM_B200_H */
