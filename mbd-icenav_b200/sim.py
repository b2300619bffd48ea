"""Host side of the drop-in: ``make_frame_step`` / ``frame_step`` / ``scan_segment``.

Mirrors the reference's interface in ``medea_ice_ship/jax_simulation.py``:

* ``make_frame_step(static, cfg, ship_dyn, ship_length, ship_beam, n_ice_steps,
  dt, dt_ice, use_auto_icenav, B_mat, T_n)`` — same arguments and meaning as
  ``_make_frame_step`` (``jax_simulation.py:302-314``); returns a callable
  ``frame_step(state, ship_state, setpoint, setpoint_next, v_water,
  dpdem_eligible, v_water_ship=None) -> (IceState, ShipState, diag)``
  (``jax_simulation.py:397-699``);
* ``FrameStep.scan_segment(state, ship_state, setpoints_K6, v_water_Kn2,
  v_water_ship_K2=None) -> (state, ship_state, histories)`` with the history
  tuple of ``JaxSimContext.scan_segment`` (``jax_simulation.py:1308-1335``);
* ``build_sim_context`` / ``run_segment`` mirror ``build_jax_sim_context`` /
  ``_run_jax_segment`` (``jax_simulation.py:1229-1384``).

Arrays are torch CUDA tensors.  Inputs given as other DLPack producers (JAX
arrays included) are wrapped with ``torch.from_dlpack`` without a copy when
they already live on the device in the right dtype and layout.  Every call is
functional: new output tensors are allocated (from torch's caching allocator)
and the inputs are not modified.  The only work done on the host is argument
marshalling; all physics runs in ``libdem_b200.so``.
"""
from __future__ import annotations

import ctypes as C
from typing import NamedTuple, Optional

import numpy as np

from . import _abi
from .config import DEFAULT_MATERIAL, IceMaterial, cfg_get
from .state import IceState, IceStaticData, ShipDynamicsData, ShipState

_torch = None


def _tm():
    global _torch
    if _torch is None:
        import torch
        _torch = torch
    return _torch


def _as_tensor(x, dtype, device):
    """Torch view of ``x`` on ``device`` with ``dtype`` (zero-copy when possible)."""
    torch = _tm()
    if x is None:
        return None
    if not isinstance(x, torch.Tensor):
        if hasattr(x, "__dlpack__") and not isinstance(x, np.ndarray):
            x = torch.from_dlpack(x)
        else:
            x = torch.as_tensor(np.asarray(x))
    if dtype is not None and x.dtype != dtype:
        x = x.to(dtype)
    if x.device != device:
        x = x.to(device)
    if not x.is_contiguous():
        x = x.contiguous()
    return x


def _ptr(t) -> Optional[int]:
    return None if t is None else int(t.data_ptr())


def _host(x) -> np.ndarray:
    if hasattr(x, "detach"):
        return x.detach().cpu().numpy().astype(np.float64)
    return np.asarray(x, dtype=np.float64)


def build_params(cfg, ship_dyn, ship_length, ship_beam, n_ice_steps, dt, dt_ice, use_auto_icenav,
                 B_mat, T_n, material: IceMaterial = DEFAULT_MATERIAL, skin: float = 0.8,
                 max_neighbors: int = 32, bucket_capacity: int = 32) -> _abi.DemParams:
    """Fill ``DemParams`` from a config the way the factory reads it (``jax_simulation.py:325-361``)."""
    P = _abi.DemParams()
    P.half_len = ship_length / 2.0
    P.half_beam = ship_beam / 2.0
    P.n_edge_samples = int(cfg_get(cfg, "n_edge_samples"))
    P.n_ice_steps = int(n_ice_steps)
    P.dt = float(dt)
    P.dt_ice = float(dt_ice)
    for name in ("bond_stiffness_factor", "hertz_factor", "hertz_exponent", "ice_ice_friction",
                 "friction_cap", "c_d_drag", "drag_ref_thickness", "linear_drag_factor",
                 "drag_coefficient_moment", "angular_damping", "pen_crit_ref",
                 "pen_crit_thickness_ref", "w_contact_cap", "w_contact_radius_factor",
                 "side_push_factor", "submergence_rate", "submergence_pen_cap", "rise_time_const",
                 "effective_strength_collision", "max_fracture_thickness", "ice_brake_threshold",
                 "bond_cohesion", "bond_internal_friction", "bond_G_c_I", "bond_G_c_II",
                 "bond_eta_bk"):
        setattr(P, name, float(cfg_get(cfg, name)))
    lo, hi = cfg_get(cfg, "angular_cap")
    P.angular_cap_lo, P.angular_cap_hi = float(lo), float(hi)
    P.velocity_clip = float(np.max(np.abs(np.asarray(cfg_get(cfg, "velocity_clip"), np.float64))))
    P.position_clip = float(cfg_get(cfg, "position_clip_m"))
    vs = [float(v) for v in cfg_get(cfg, "ship_velocity_clip")]
    P.vc_surge, P.vc_sway, P.vc_yaw = vs
    mx = cfg_get(cfg, "max_ship_ice_force")
    P.has_max_ship_ice_force = 0 if mx is None else 1
    P.max_ship_ice_force = 0.0 if mx is None else float(mx)
    P.use_auto_icenav = 1 if use_auto_icenav else 0
    P.youngs_modulus = float(material.youngs_modulus)
    P.water_density = float(material.water_density)
    P.flexural_strength_base = float(material.flexural_strength_base)
    P.T_n = float(T_n)
    for name, arr, size in (("B_mat", B_mat, 18), ("M3inv", ship_dyn.M3inv, 9), ("D3", ship_dyn.D3, 9),
                            ("Kp", ship_dyn.Kp, 9), ("Kd", ship_dyn.Kd, 9), ("Ki", ship_dyn.Ki, 9),
                            ("B_pinv", ship_dyn.B_pinv, 18), ("n_max", ship_dyn.n_max, 6)):
        v = _host(arr).reshape(-1)
        if v.size != size:
            raise ValueError(f"{name} has {v.size} entries, expected {size}")
        setattr(P, name, (C.c_double * size)(*v.tolist()))
    P.skin = float(skin)
    P.max_neighbors = int(max_neighbors)
    P.bucket_capacity = int(bucket_capacity)
    return P


class FrameStep:
    """Compiled-once frame step bound to one ice field (what ``make_frame_step`` returns)."""

    def __init__(self, static: IceStaticData, cfg, ship_dyn: ShipDynamicsData, ship_length: float,
                 ship_beam: float, n_ice_steps: int, dt: float, dt_ice: float,
                 use_auto_icenav: bool, B_mat, T_n: float, material: IceMaterial = DEFAULT_MATERIAL,
                 skin: float = 0.8, max_neighbors: int = 32, bucket_capacity: int = 32,
                 device=None, dtype=None, launch_mode: int = _abi.DEM_LAUNCH_PERSISTENT,
                 system_start=None):
        """``system_start`` (Q+1 element offsets) splits the field into Q independent
        systems, each with its own ship; they step together through ``scan_segment``
        with ship arrays of shape (Q, 3) / (Q, 6) and setpoints of shape (K, Q, 6)."""
        torch = _tm()
        self.lib = _abi.load_library()
        if device is None:
            device = static.masses.device if hasattr(static.masses, "device") else torch.device("cuda", torch.cuda.current_device())
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise ValueError("the DEM frame step runs on a CUDA device only")
        if dtype is None:
            m = static.masses
            dtype = m.dtype if hasattr(m, "dtype") and isinstance(m, torch.Tensor) else torch.float32
        if dtype not in (torch.float32, torch.float64):
            raise ValueError("dtype must be float32 or float64")
        self.dtype = dtype
        dev, dt_ = self.device, dtype
        f = lambda x: _as_tensor(x, dt_, dev)
        i32 = lambda x: _as_tensor(x, torch.int32, dev)
        u8 = lambda x: _as_tensor(x, torch.bool, dev).view(torch.uint8)
        if static.pair_i is not None and static.pair_j is not None:
            n_ = int(static.masses.shape[0])
            if int(np.prod(static.pair_i.shape)) != n_ * (n_ - 1) // 2:
                raise ValueError("pair_i/pair_j must be the full upper-triangle list; the GPU broad "
                                 "phase resolves all pairs")
        self._keep = dict(
            polys=f(static.local_polys_padded), mask=u8(static.poly_mask), nverts=i32(static.poly_n_verts),
            masses=f(static.masses), inertia=f(static.inertia), radii=f(static.radii), areas=f(static.areas),
            thick=f(static.thicknesses), bi=i32(static.bond_i), bj=i32(static.bond_j),
            rest=f(static.rest_lengths), bstr=f(static.bond_strengths), sbar=f(static.sigma_bar_bond),
            floe=i32(static.initial_floe_of), hull=f(ship_dyn.ship_hull_local))
        k = self._keep
        self.n = int(k["masses"].shape[0])
        self.n_bonds = int(k["bi"].shape[0])
        self.max_v = int(k["polys"].shape[1])
        self.n_floes = int(k["floe"].max().item()) + 1 if self.n else 0
        S = _abi.DemStatic()
        S.n, S.max_v, S.n_bonds, S.n_floes = self.n, self.max_v, self.n_bonds, self.n_floes
        S.n_hull = int(k["hull"].shape[0])
        S.local_polys_padded = _ptr(k["polys"])
        S.poly_mask = _ptr(k["mask"])
        S.poly_n_verts = _ptr(k["nverts"])
        S.masses, S.inertia, S.radii = _ptr(k["masses"]), _ptr(k["inertia"]), _ptr(k["radii"])
        S.areas, S.thicknesses = _ptr(k["areas"]), _ptr(k["thick"])
        S.bond_i, S.bond_j = _ptr(k["bi"]), _ptr(k["bj"])
        S.rest_lengths, S.bond_strengths = _ptr(k["rest"]), _ptr(k["bstr"])
        S.sigma_bar_bond, S.initial_floe_of = _ptr(k["sbar"]), _ptr(k["floe"])
        S.k_n, S.k_s = float(static.k_n), float(static.k_s)
        S.ship_hull_local = _ptr(k["hull"])
        self.n_systems = 1
        if system_start is not None and len(system_start) > 2:
            self.n_systems = len(system_start) - 1
            self._sys_start = (C.c_int32 * len(system_start))(*[int(v) for v in system_start])
            S.n_systems = self.n_systems
            S.system_start = C.cast(self._sys_start, C.POINTER(C.c_int32))
        self.params = build_params(cfg, ship_dyn, ship_length, ship_beam, n_ice_steps, dt, dt_ice,
                                   use_auto_icenav, B_mat, T_n, material, skin, max_neighbors,
                                   bucket_capacity)
        self.n_ice_steps = int(n_ice_steps)
        self.dt = float(dt)
        h = C.c_void_p()
        with torch.cuda.device(self.device):
            torch.cuda.synchronize()
            rc = self.lib.dem_create(C.byref(self.params), C.byref(S),
                                     _abi.DEM_F64 if dtype == torch.float64 else _abi.DEM_F32,
                                     self.device.index if self.device.index is not None else torch.cuda.current_device(),
                                     C.byref(h))
        self._h = h
        if rc != _abi.DEM_OK:
            msg = self._error()
            self.lib.dem_destroy(h)
            self._h = None
            raise _abi.DemError(rc, msg)
        if launch_mode != _abi.DEM_LAUNCH_PERSISTENT:
            self.set_launch_mode(launch_mode)

    # ── housekeeping ──────────────────────────────────────────────────────────
    def _error(self) -> str:
        buf = C.create_string_buffer(512)
        if self._h:
            self.lib.dem_get_error(self._h, buf, 512)
        return buf.value.decode(errors="replace")

    def _check(self, rc):
        if rc != _abi.DEM_OK:
            raise _abi.DemError(rc, self._error())

    def set_launch_mode(self, mode: int):
        self._check(self.lib.dem_set_launch_mode(self._h, int(mode)))

    def set_work_split(self, force_split: int = 0, mark_split: int = 0):
        """How substep work is split (``dem_set_work_split``; results are identical)."""
        self._check(self.lib.dem_set_work_split(self._h, int(force_split), int(mark_split)))

    def info(self) -> dict:
        inf = _abi.DemInfo()
        self._check(self.lib.dem_get_info(self._h, C.byref(inf)))
        return {k: getattr(inf, k) for k, _ in _abi.DemInfo._fields_}

    def set_profiling(self, on: bool = True):
        """Record device time stamps at every phase end of persistent launches."""
        self._check(self.lib.dem_set_profiling(self._h, 1 if on else 0))

    def phase_times(self):
        """[(phase index, ns since launch start)] of the last profiled persistent call."""
        buf = (C.c_int64 * (2 * 4096))()
        cnt = C.c_int32()
        t0 = C.c_int64()
        self._check(self.lib.dem_get_phase_times(self._h, buf, 4096, C.byref(cnt), C.byref(t0)))
        return [(int(buf[2 * i]), int(buf[2 * i + 1]) - int(t0.value)) for i in range(cnt.value)]

    def record_contacts(self, capacity: int = 1 << 20, max_marks: int = 4096) -> "ContactRecorder":
        """Record the ice-ice contact set of every later call (``dem_debug_record_contacts``):
        the pairs whose contact term each substep's force phase computed.  Returns
        the recorder; ``stop_recording`` turns it off."""
        rec = ContactRecorder(self.device, capacity, max_marks)
        self._check(self.lib.dem_debug_record_contacts(self._h, _ptr(rec.pairs), capacity, _ptr(rec.marks),
                                                       max_marks, _ptr(rec.count)))
        self._recorder = rec
        return rec

    def stop_recording(self):
        self._check(self.lib.dem_debug_record_contacts(self._h, None, 0, None, 0, None))
        self._recorder = None

    def close(self):
        if getattr(self, "_h", None):
            self.lib.dem_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _stream(self):
        return C.c_void_p(_tm().cuda.current_stream(self.device).cuda_stream)

    # ── state marshalling ─────────────────────────────────────────────────────
    def _ice_in(self, state: IceState):
        torch = _tm()
        f = lambda x: _as_tensor(x, self.dtype, self.device)
        b = lambda x: _as_tensor(x, torch.bool, self.device)
        return IceState(positions=f(state.positions), velocities=f(state.velocities),
                        rotations=f(state.rotations), angular_vels=f(state.angular_vels),
                        submergence=f(state.submergence), bond_intact=b(state.bond_intact),
                        bond_damage=f(state.bond_damage), bond_delta_m_0=f(state.bond_delta_m_0),
                        bond_delta_m_max=f(state.bond_delta_m_max), bond_delta_s=f(state.bond_delta_s),
                        elem_active=b(state.elem_active), dpdem_floe_eligible=b(state.dpdem_floe_eligible))

    def _ship_in(self, ship: ShipState):
        f = lambda x: _as_tensor(x, self.dtype, self.device)
        return ShipState(eta=f(ship.eta), nu=f(ship.nu), n_actual=f(ship.n_actual), e_int=f(ship.e_int))

    def _alloc_state(self) -> IceState:
        torch = _tm()
        n, nb, nf, d, dev = self.n, self.n_bonds, self.n_floes, self.dtype, self.device
        e = lambda *s: torch.empty(s, dtype=d, device=dev)
        eb = lambda *s: torch.empty(s, dtype=torch.bool, device=dev)
        return IceState(positions=e(n, 2), velocities=e(n, 2), rotations=e(n), angular_vels=e(n),
                        submergence=e(n), bond_intact=eb(nb), bond_damage=e(nb), bond_delta_m_0=e(nb),
                        bond_delta_m_max=e(nb), bond_delta_s=e(nb), elem_active=eb(n),
                        dpdem_floe_eligible=eb(nf))

    def _alloc_ship(self) -> ShipState:
        torch = _tm()
        qs = () if self.n_systems == 1 else (self.n_systems,)
        e = lambda k: torch.empty(qs + (k,), dtype=self.dtype, device=self.device)
        return ShipState(eta=e(3), nu=e(3), n_actual=e(6), e_int=e(3))

    @staticmethod
    def _c_state(st: IceState) -> _abi.DemIceState:
        c = _abi.DemIceState()
        for name in IceState._fields:
            setattr(c, name, _ptr(getattr(st, name)))
        return c

    @staticmethod
    def _c_ship(sh: ShipState) -> _abi.DemShipState:
        c = _abi.DemShipState()
        for name in ShipState._fields:
            setattr(c, name, _ptr(getattr(sh, name)))
        return c

    def _run(self, fn, *args, retries: int = 4, check: bool = True):
        for attempt in range(retries + 1):
            self._check(fn(self._h, *args))
            if not check:
                return
            rc = self.lib.dem_sync_status(self._h, self._stream())
            if rc == _abi.DEM_OK:
                return
            if rc == _abi.DEM_ERR_CAPACITY and attempt < retries and self.grow_capacity():
                continue  # inputs are untouched: run the same call again
            raise _abi.DemError(rc, self._error())

    def grow_capacity(self) -> bool:
        """After ``DEM_ERR_CAPACITY``: enlarge what overflowed (neighbour lists up
        to 64 entries, grid buckets without limit) and reset the broad phase.
        Returns False when nothing can grow any more."""
        flags = self.info()["capacity_flags"] or 3
        P = self.params
        nb, bc = P.max_neighbors, P.bucket_capacity
        if flags & 2:
            nb = min(64, int(nb * 1.5) + 1)
        if flags & 1:
            bc = int(bc * 2)
        if (nb, bc) == (P.max_neighbors, P.bucket_capacity):
            return False
        P.max_neighbors, P.bucket_capacity = nb, bc
        self._check(self.lib.dem_set_capacity(self._h, nb, bc))
        return True

    # ── the reference-facing calls ────────────────────────────────────────────
    def __call__(self, state: IceState, ship_state: ShipState, setpoint, setpoint_next, v_water,
                 dpdem_eligible, v_water_ship=None, check: bool = True):
        """One frame (``frame_step``, ``jax_simulation.py:397-699``)."""
        torch = _tm()
        st = self._ice_in(state)
        sh = self._ship_in(ship_state)
        f = lambda x: _as_tensor(x, self.dtype, self.device)
        sp, spn, vw = f(setpoint), f(setpoint_next), f(v_water)
        el = _as_tensor(dpdem_eligible, torch.bool, self.device)
        vws = None if v_water_ship is None else f(v_water_ship)
        if vw.shape != (self.n, 2):
            raise ValueError(f"v_water must be ({self.n}, 2)")
        out = self._alloc_state()
        sh_out = self._alloc_ship()
        diag_t = dict(pen_max=torch.empty(self.n, dtype=self.dtype, device=self.device),
                      force_mag=torch.empty(self.n, dtype=self.dtype, device=self.device),
                      F_ice_on_ship=torch.empty(2, dtype=self.dtype, device=self.device),
                      J_cumul_incr=torch.empty((), dtype=self.dtype, device=self.device))
        cdiag = _abi.DemDiag(*[_ptr(diag_t[k]) for k, _ in _abi.DemDiag._fields_])
        cin, cout = self._c_state(st), self._c_state(out)
        sin, sout = self._c_ship(sh), self._c_ship(sh_out)
        self._run(self.lib.dem_frame_step, C.byref(cin), C.byref(cout), C.byref(sin), C.byref(sout),
                  _ptr(sp), _ptr(spn), _ptr(vw), _ptr(el), _ptr(vws), C.byref(cdiag), self._stream(),
                  check=check)
        return out, sh_out, diag_t

    def scan_segment(self, state: IceState, ship_state: ShipState, setpoints_K6, v_water_Kn2,
                     v_water_ship_K2=None, history: bool = True, check: bool = True):
        """K frames in one launch (``JaxSimContext.scan_segment``, ``jax_simulation.py:1308-1335``).

        Returns ``(final_state, final_ship, (positions (K,n,2), rotations (K,n),
        bond_intact (K,n_bonds), eta (K,3), submergence (K,n), J_cumul_incr (K,),
        F_ice_on_ship (K,2)))``; with ``history=False`` the tuple is ``None``, with
        ``history="ship"`` only eta, J_cumul_incr and F_ice_on_ship are recorded
        (the ice rows are ``None``).  With Q systems the per-ship arrays gain a
        (Q,) axis after K.
        """
        return self._segment(self.lib.dem_scan_segment, 6, state, ship_state, setpoints_K6, v_water_Kn2,
                             v_water_ship_K2, history, check)

    def rollout_segment(self, state: IceState, ship_state: ShipState, controls_K3, v_water_Kn2,
                        v_water_ship_K2=None, history: bool = True, check: bool = True):
        """K frames with every ship driven by body-frame controls [X, Y, N] instead of
        setpoints (``dem_rollout_segment``): ``controls_K3`` is (K, 3), or (K, Q, 3) with
        Q systems.  Returns what ``scan_segment`` returns."""
        return self._segment(self.lib.dem_rollout_segment, 3, state, ship_state, controls_K3, v_water_Kn2,
                             v_water_ship_K2, history, check)

    def alloc_history(self, K: int, history=True):
        """Device buffers of ``K`` frames' history rows in the order of the
        C ABI's ``DemHistory``: (pos, rot, intact, eta, submergence,
        J_cumul_incr, F_ice_on_ship); ``history="ship"`` leaves the ice rows
        out (``None``)."""
        torch = _tm()
        if history not in (True, "ship"):
            raise ValueError("history must be True, False or 'ship'")
        d, dev = self.dtype, self.device
        qs = () if self.n_systems == 1 else (self.n_systems,)
        ice = history is True
        return (torch.empty((K, self.n, 2), dtype=d, device=dev) if ice else None,
                torch.empty((K, self.n), dtype=d, device=dev) if ice else None,
                torch.empty((K, self.n_bonds), dtype=torch.bool, device=dev) if ice else None,
                torch.empty((K,) + qs + (3,), dtype=d, device=dev),
                torch.empty((K, self.n), dtype=d, device=dev) if ice else None,
                torch.empty((K,) + qs, dtype=d, device=dev),
                torch.empty((K,) + qs + (2,), dtype=d, device=dev))

    def _segment(self, fn, row_len, state, ship_state, rows_K, v_water_Kn2, v_water_ship_K2, history, check):
        torch = _tm()
        st = self._ice_in(state)
        sh = self._ship_in(ship_state)
        f = lambda x: _as_tensor(x, self.dtype, self.device)
        sp = f(rows_K)
        vw = f(v_water_Kn2)
        K = int(sp.shape[0])
        Q = self.n_systems
        qs = () if Q == 1 else (Q,)
        if tuple(sp.shape) != (K,) + qs + (row_len,) or vw.shape != (K, self.n, 2):
            raise ValueError(f"per-frame rows must be {(K,) + qs + (row_len,)} and v_water_Kn2 (K,n,2)")
        vws = None if v_water_ship_K2 is None else f(v_water_ship_K2)
        out = self._alloc_state()
        sh_out = self._alloc_ship()
        hist = None
        chist = None
        if history:
            hist = self.alloc_history(K, history)
            chist = _abi.DemHistory(*[_ptr(t) for t in hist])
        cin, cout = self._c_state(st), self._c_state(out)
        sin, sout = self._c_ship(sh), self._c_ship(sh_out)
        self._run(fn, C.byref(cin), C.byref(cout), C.byref(sin), C.byref(sout), K, _ptr(sp), _ptr(vw), _ptr(vws),
                  C.byref(chist) if chist is not None else None, self._stream(), check=check)
        return out, sh_out, hist


class ContactRecorder:
    """Device buffers of ``dem_debug_record_contacts`` and their readout."""

    def __init__(self, device, capacity: int, max_marks: int):
        torch = _tm()
        self.pairs = torch.zeros((max(capacity, 1), 2), dtype=torch.int32, device=device)
        self.marks = torch.zeros(max(max_marks, 1), dtype=torch.int32, device=device)
        self.count = torch.zeros(1, dtype=torch.int32, device=device)  # read as uint32
        self.capacity = capacity

    def substeps(self, n_substeps: int):
        """Pairs of each substep of the last call, as (i < j) sets: a list of
        ``n_substeps`` sets of tuples, and the raw {e, o} records per substep."""
        _tm().cuda.synchronize()
        total = int(self.count.item()) & 0xFFFFFFFF
        if total > self.capacity:
            raise RuntimeError(f"contact recorder overflow: {total} pairs > capacity {self.capacity}")
        marks = self.marks[:n_substeps].cpu().numpy().astype(np.int64)
        pairs = self.pairs[:total].cpu().numpy().astype(np.int64)
        sets, raw = [], []
        lo = 0
        for m in marks:
            p = pairs[lo:m]
            raw.append(p)
            sets.append(set(zip(np.minimum(p[:, 0], p[:, 1]).tolist(), np.maximum(p[:, 0], p[:, 1]).tolist())))
            lo = int(m)
        return sets, raw


def make_frame_step(static, cfg, ship_dyn, ship_length, ship_beam, n_ice_steps, dt, dt_ice,
                    use_auto_icenav, B_mat, T_n, **kw) -> FrameStep:
    """Drop-in for ``_make_frame_step`` (``jax_simulation.py:302-314``)."""
    return FrameStep(static, cfg, ship_dyn, ship_length, ship_beam, n_ice_steps, dt, dt_ice,
                     use_auto_icenav, B_mat, T_n, **kw)


class SimContext(NamedTuple):
    """Mirror of ``JaxSimContext`` (``jax_simulation.py:1211-1226``)."""

    frame_step: FrameStep
    scan_segment: object
    static: IceStaticData
    ship_dyn: ShipDynamicsData
    n: int
    n_bonds: int
    dt: float
    chunk_size: int


def substep_count(static_radii, cfg, dt, material: IceMaterial = DEFAULT_MATERIAL):
    """(dt_ice, n_ice_steps) with the optional Rayleigh cap (``jax_simulation.py:1258-1281``)."""
    nu_r = cfg_get(cfg, "poisson_ratio")
    G = material.youngs_modulus / (2.0 * (1.0 + nu_r))
    r_min = float(np.min(_host(static_radii)))
    b = cfg_get(cfg, "rayleigh_safety_factor")
    dt_r = b * np.pi * r_min / (0.163 * nu_r + 0.877) * np.sqrt(material.ice_density / G)
    dt_ice = min(dt, dt_r) if cfg_get(cfg, "use_rayleigh_dt_cap") else dt
    n_steps = max(1, int(round(dt / dt_ice))) if dt_ice > 0 else 1
    return dt_ice, n_steps


def build_sim_context(polygons, centroids, bonds, ship_pos, ship_length, ship_beam, n_frames, dt,
                      drift_vel, thicknesses, ship_props, config=None, parent_ids=None,
                      use_auto_icenav_ship: bool = False, chunk_size: int = 50, verbose: bool = True,
                      n_ice_steps: Optional[int] = None, material: IceMaterial = DEFAULT_MATERIAL,
                      dilation: float = 0.0, hull_local=None, dtype=None, device="cuda",
                      **frame_kw) -> SimContext:
    """Mirror of ``build_jax_sim_context`` (``jax_simulation.py:1229-1358``).

    ``n_ice_steps`` overrides the substep count the config implies (the
    reference reaches a given count through the factory arguments).
    """
    from .config import get_default_simulation_config
    from .state import build_ship_dynamics_data, build_static_data
    from .vessel import SupplyVessel

    cfg = config or get_default_simulation_config()
    static = build_static_data(polygons, centroids, bonds, thicknesses, parent_ids, cfg, material,
                               dilation, dtype, device)
    ship_dyn = build_ship_dynamics_data(ship_props, cfg, ship_length, ship_beam, hull_local, dtype, device)
    if n_ice_steps is None:
        dt_ice, k = substep_count(static.radii, cfg, dt, material)
    else:
        k = int(n_ice_steps)
        dt_ice = dt / k
    sv = SupplyVessel(mass=ship_props.mass, length=ship_length)
    fs = make_frame_step(static, cfg, ship_dyn, ship_length, ship_beam, k, dt, dt_ice,
                         use_auto_icenav_ship, sv.B, sv.T_n, material=material, **frame_kw)
    if verbose:
        print(f"  [DEM] frame step ready: {fs.n} elements, {fs.n_bonds} bonds, {k} substeps", flush=True)
    return SimContext(frame_step=fs, scan_segment=fs.scan_segment, static=static, ship_dyn=ship_dyn,
                      n=fs.n, n_bonds=fs.n_bonds, dt=float(dt), chunk_size=int(chunk_size))


def run_segment(ctx: SimContext, state, ship_state, setpoints_K6, v_water_Kn2, v_water_ship_K2=None):
    """Mirror of ``_run_jax_segment`` (``jax_simulation.py:1361-1384``)."""
    return ctx.scan_segment(state, ship_state, setpoints_K6, v_water_Kn2, v_water_ship_K2)
