#!/usr/bin/env python
"""Throughput of the plain-DEM frame step (DEM element-steps/s) on one B200 per rank.

Workload: the large seeded field (1.5 x 1.5 km at ~70 %, power-law floes
tessellated into ~245k elements, ~826k bonds, dilation 0.05 m), 7-vertex
60 x 12 m hull on a piecewise-linear path at 2.5 m/s, 10 substeps of 0.005 s
per 0.05 s frame, fp32.  A step is one frame (10 substeps) of the whole
field; ``--steps`` defaults to 1000 frames = the workload's 10,000 substeps.

* ``value``        element-steps/s = n * substeps * frames / device time, inputs
                   resident in HBM, L2 flushed (256 MB write) before every frame,
                   each frame timed with CUDA events on the launch stream;
* ``e2e``          the same metric through the public API (``scan_segment``) with
                   host buffers: per frame the setpoint row and v_water (n,2) are
                   copied from pinned host memory and the frame's history (positions,
                   rotations, bond_intact, eta, submergence, J, F) is copied back;
                   L2 flushed before every frame; the median of three timed windows;
* ``roofline``     algorithmic bytes per frame / mean frame time vs measured HBM;
* ``cpu_baseline`` the NumPy oracle (float64, restated broad phase) on a window
                   of the same field, on this host, one core.

``--impl reference`` times the oracle port alone (the reference itself is JAX,
which this image cannot run) with a process per host core, each on its own
window of the field.  Multi-GPU (torchrun) runs independent replicas, one per
rank ("scaling": "weak"); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "mbd-icenav_b200"))

METRIC = "DEM elem-steps/s"
UNIT = "elem-steps/s"
N_SUB = 10
DT = 0.05
START_FRAME = 400  # the ship is ~60 m into the field by then, so contacts occur
E2E_WARMUP = 3  # untimed end-to-end steps before the timed ones
E2E_WINDOWS = 3  # timed end-to-end windows (the median is reported)


def _abi_mod():
    _pkg()
    from mbd_icenav_b200 import _abi
    return _abi


def _pkg():
    import _pkg as loader
    return loader.load_package()


def cache_dir():
    d = os.environ.get("MBD_ICENAV_CACHE", "/tmp/mbd_icenav_b200_cache")
    os.makedirs(d, exist_ok=True)
    return d


def load_field(name: str, seed: int):
    """Seeded field, cached as .npz for later runs in the same container."""
    import numpy as np
    from mbd_icenav_b200 import scene
    path = os.path.join(cache_dir(), f"{name}_{seed}.npz")
    if os.path.exists(path):
        z = np.load(path, allow_pickle=False)
        offs = z["poly_off"]
        verts = z["poly_verts"]
        polys = [verts[offs[i]:offs[i + 1]] for i in range(len(offs) - 1)]
        f = scene.make_field.__globals__["IceField"](
            name=name, polygons=polys, centroids=z["centroids"], bonds=[tuple(b) for b in z["bonds"].tolist()],
            thicknesses=z["thicknesses"], parent_ids=z["parent_ids"], ship_length=float(z["ship"][0]),
            ship_beam=float(z["ship"][1]),
            ship_props=scene.ShipProperties(length=float(z["ship"][0]), beam=float(z["ship"][1]), draft=4.0),
            hull_local=z["hull"], trajectory=z["trajectory"], current=tuple(z["current"].tolist()),
            dt=DT, n_ice_steps=N_SUB, n_frames=len(z["trajectory"]) - 2, domain=tuple(z["domain"].tolist()))
        return f
    f = scene.make_field(name, seed=seed, n_frames=START_FRAME + 3000)
    offs = np.cumsum([0] + [len(p) for p in f.polygons])
    np.savez(path + ".tmp.npz", poly_off=offs, poly_verts=np.concatenate(f.polygons), centroids=f.centroids,
             bonds=np.array(f.bonds, np.int64), thicknesses=f.thicknesses, parent_ids=f.parent_ids,
             ship=np.array([f.ship_length, f.ship_beam]), hull=f.hull_local, trajectory=f.trajectory,
             current=np.array(f.current), domain=np.array(f.domain))
    os.replace(path + ".tmp.npz", path)
    return f


def algorithmic_bytes_per_frame(n: int, nb: int, V: int, k: int, n_act=None, nb_act=None, in_place=False) -> int:
    """Bytes each frame must move at minimum, fp32, bool = 1 B, i32 = 4 B.

    Per substep and active element: read pos 8 + vel 8 + rot 4 + w 4 + sub 4 +
    active 1 + mass 4 + inertia 4 + radius 4 + area 4 + thickness 4 + ship force
    8 + v_water 8, write pos 8 + vel 8 + rot 4 + w 4 = 89 B.  A frozen element
    keeps its state whatever its forces (jax_simulation.py:257-262), so it only
    carries it over from the frame's input to its output, once per frame: read
    pos, vel, rot, w, active, write pos, vel, rot, w = 49 B.  Per substep and
    bond with an active end: i 4 + j 4 + rest length 4 + damage 4 + intact 1 =
    17 B (a bond between two frozen elements is not read).  Per frame: ship
    contact n (9V + 64) B and the bond update 50 B per bond.  ``n_act`` /
    ``nb_act`` default to n / nb (every element active).  ``in_place``: a frame
    after the first of a multi-frame call, which updates the state in place, so
    frozen elements have nothing to carry over.
    """
    n_act = n if n_act is None else n_act
    nb_act = nb if nb_act is None else nb_act
    carry = 0 if in_place else 49 * (n - n_act)
    return int(k * (89 * n_act + 17 * nb_act) + carry + n * (9 * V + 64) + 50 * nb)


def active_counts(elem_active, bond_i, bond_j):
    """(active elements, bonds with an active end) of a state, on the device."""
    a = elem_active.bool()
    return int(a.sum().item()), int((a[bond_i.long()] | a[bond_j.long()]).sum().item())


def peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def committed_traffic(workload: str):
    """Per-launch DRAM bytes of the frame kernel from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return d.get(workload)
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join(cache_dir(), f"clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
            # nvidia-smi's first query can hold the GPU up for a while: let it
            # complete (first sample written, 5 s at most) before the timed region
            t0 = time.time()
            while time.time() - t0 < 5.0 and os.path.getsize(self.path) == 0 and self.proc.poll() is None:
                time.sleep(0.05)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        import statistics
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                rows.append((float(p[1]), float(p[2]), float(p[3]), p[5], p[6], p[7], p[8]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        reasons = set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            for nm, v in zip(names, r[3:]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "power_w_max": max(r[2] for r in rows), "samples": len(rows), "reasons": sorted(reasons)}


def build_stepper(field, dtype_name: str, device, bucket_capacity: int = 64, skin: float = 0.8):
    import numpy as np
    import torch
    from mbd_icenav_b200 import sim
    from mbd_icenav_b200.config import SimulationConfig
    from mbd_icenav_b200.state import (build_ship_dynamics_data, build_static_data,
                                       initial_ice_state_arrays, initial_ship_state_arrays, to_device)
    from mbd_icenav_b200.vessel import SupplyVessel
    dt = torch.float32 if dtype_name == "f32" else torch.float64
    cfg = SimulationConfig()
    static = build_static_data(field.polygons, field.centroids, field.bonds, field.thicknesses,
                               field.parent_ids, cfg, dilation=0.05, dtype=dt, device=device)
    sdyn = build_ship_dynamics_data(field.ship_props, cfg, field.ship_length, field.ship_beam,
                                    field.hull_local, dtype=dt, device=device)
    sv = SupplyVessel(mass=field.ship_props.mass, length=field.ship_length)
    fs = sim.make_frame_step(static, cfg, sdyn, field.ship_length, field.ship_beam, N_SUB, DT, DT / N_SUB,
                             False, sv.B, sv.T_n, device=device, dtype=dt, bucket_capacity=bucket_capacity,
                             skin=skin)
    st = to_device(initial_ice_state_arrays(field.n, field.centroids, len(field.bonds), field.parent_ids), dt, device)
    eta0 = field.trajectory[START_FRAME]
    sh = to_device(initial_ship_state_arrays(eta0[:2], float(eta0[2])), dt, device)
    return fs, st, sh, static


class DirectFrames:
    """Single-frame ``dem_scan_segment`` calls through the C ABI on two
    preallocated state buffers (frame i reads buffer i % 2 and writes the
    other), with the argument structs built once: nothing is allocated or
    marshalled between two frames, so a timed frame holds device work only."""

    def __init__(self, fs, sp_all, vw):
        import ctypes as C
        self.C = C
        self.fs = fs
        self.bufs = [(fs._alloc_state(), fs._alloc_ship()) for _ in range(2)]
        self.c_ice = [fs._c_state(b[0]) for b in self.bufs]
        self.c_ship = [fs._c_ship(b[1]) for b in self.bufs]
        self.sp_all = sp_all  # (F, 6), row f = frame f's setpoints
        self.sp_base = int(sp_all.data_ptr())
        self.sp_row = 6 * sp_all.element_size()
        self.vw_ptr = C.c_void_p(int(vw.data_ptr()))
        self.stream = fs._stream()
        self.cur = 0  # buffer holding the current state

    def load(self, st, sh):
        """Copy a state into the current buffer (outside any timed region)."""
        ice, ship = self.bufs[self.cur]
        for dst, src in zip(ice, st):
            dst.copy_(src)
        for dst, src in zip(ship, sh):
            dst.copy_(src)

    def state(self):
        return self.bufs[self.cur]

    def frame(self, fr: int, io=None):
        """Enqueue one frame with setpoint row ``fr``; returns the call's status.
        ``io = (setpoints, v_water, history)``: the frame reads its setpoint row
        and field from those device pointers instead and writes its history
        rows through that ``DemHistory``."""
        C, a, b = self.C, self.cur, 1 - self.cur
        if io is None:
            sp, vw, hist = C.c_void_p(self.sp_base + fr * self.sp_row), self.vw_ptr, None
        else:
            sp, vw, hist = io[0], io[1], C.byref(io[2])
        rc = self.fs.lib.dem_scan_segment(self.fs._h, C.byref(self.c_ice[a]), C.byref(self.c_ice[b]),
                                          C.byref(self.c_ship[a]), C.byref(self.c_ship[b]), 1, sp, vw, None,
                                          hist, self.stream)
        self.cur = b
        return rc


def host_head_start(frames: int):
    """A device sleep long enough for the host to enqueue `frames` timed frames
    (flush, two events and one library call each, ~60 us of host time) before
    the GPU reaches the first: every event pair then brackets device work only."""
    import torch
    ms = min(200.0, 5.0 + 0.06 * frames)
    torch.cuda._sleep(int(ms * 2.0e6))  # ~2 GHz SM clock


def max_over_ranks(seconds: float, world: int, device) -> float:
    """The slowest rank's time: every rank calls this with its own timed seconds."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def retry_verdict(rc: int, grown: bool, world: int, device) -> int:
    """One decision for all ranks after a timed region: 0 = every rank clean,
    1 = some rank grew its capacity (all ranks time the region again),
    2 = some rank failed for good (all ranks stop)."""
    import torch
    import torch.distributed as dist
    v = torch.tensor([0.0 if rc == 0 else (1.0 if grown else 2.0)], device=device)
    if world > 1:
        dist.all_reduce(v, op=dist.ReduceOp.MAX)
    return int(v.item())


def run_ours(args, rank: int, world: int):
    import numpy as np
    import torch
    import torch.distributed as dist
    _pkg()
    device = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(device)
    field = load_field(args.config, args.seed)
    if args.order == "morton":
        from mbd_icenav_b200 import scene
        field = scene.spatially_sorted(field)
    fs, st, sh, static = build_stepper(field, args.dtype, device, args.bucket_capacity, args.skin)
    if args.launch == "phased":
        from mbd_icenav_b200 import _abi
        fs.set_launch_mode(_abi.DEM_LAUNCH_PHASED)
    dt = fs.dtype
    n, nb, V = fs.n, fs.n_bonds, fs.max_v
    K, W = args.steps, args.warmup
    total_frames = W + K + E2E_WARMUP + E2E_WINDOWS * args.e2e_steps + 1  # + the untimed end-to-end steps
    sp_all = torch.as_tensor(field.setpoints(START_FRAME, total_frames), dtype=dt, device=device)
    vw = torch.zeros((1, n, 2), dtype=dt, device=device)
    vw[0, :, 0] = float(field.current[0])
    vw[0, :, 1] = float(field.current[1])
    stream = torch.cuda.current_stream(device)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=device)

    if args.all_active:
        # every element and floe active from the start: the force path then
        # runs on the whole field each substep (the bandwidth-bound case)
        st = st._replace(elem_active=torch.ones_like(st.elem_active),
                         dpdem_floe_eligible=torch.ones_like(st.dpdem_floe_eligible))
    fr = 0
    for _ in range(W):
        st, sh, _ = fs.scan_segment(st, sh, sp_all[fr:fr + 1], vw, history=False)
        fr += 1
    direct = DirectFrames(fs, sp_all, vw)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    st_w, sh_w, fr_w = st, sh, fr
    act0 = active_counts(st.elem_active, static.bond_i, static.bond_j)
    for attempt in range(4):
        # the device status is read once after the timed frames; a capacity
        # overflow grows the scratch and times the same frames again (every rank
        # takes part, so the ranks stay in step)
        fr = fr_w
        direct.load(st_w, sh_w)
        with ClockSampler(device.index) as clk:
            torch.cuda.synchronize()
            host_head_start(K)
            for i in range(K):
                flush.fill_(i & 0xFF)  # evict L2 (126 MB) before every timed frame
                starts[i].record(stream)
                rc_call = direct.frame(fr)
                ends[i].record(stream)
                if rc_call != 0:
                    raise RuntimeError(f"dem_scan_segment returned {rc_call}: {fs._error()}")
                fr += 1
            torch.cuda.synchronize()
        rc = fs.lib.dem_sync_status(fs._h, fs._stream())
        msg = fs._error() if rc != 0 else ""
        grown = rc == _abi_mod().DEM_ERR_CAPACITY and attempt < 3 and fs.grow_capacity()
        verdict = retry_verdict(rc, grown, world, device)
        if verdict == 0:
            break
        if verdict == 2:
            raise RuntimeError(f"device status {rc}: {msg}" if rc else "device error on another rank")
    if world > 1:
        dist.barrier()
    st, sh = direct.state()
    act1 = active_counts(st.elem_active, static.bond_i, static.bond_j)
    n_act, nb_act = 0.5 * (act0[0] + act1[0]), 0.5 * (act0[1] + act1[1])
    frame_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    # the K timed frames in three consecutive windows: the reported frame time
    # is the median window's mean, so one disturbed stretch does not decide it
    nwin = 3 if K >= 3 else 1
    bounds = [round(K * w / nwin) for w in range(nwin + 1)]
    win_ms = [sum(frame_ms[bounds[w]:bounds[w + 1]]) / max(bounds[w + 1] - bounds[w], 1) for w in range(nwin)]
    frame_s = sorted(win_ms)[nwin // 2] / 1e3
    frame_max = max_over_ranks(frame_s, world, device)
    total_max = frame_max * K
    value = world * n * N_SUB / frame_max

    # end to end through the C ABI with host buffers: every step uploads its
    # setpoint row and current field from pinned host memory, runs one
    # dem_scan_segment frame and downloads its history rows, all inside the
    # timed region.  A copy stream overlaps the upload of step i+1 and the
    # download of step i-1 with step i (inputs and history rows are
    # double-buffered on the device, results on the host).
    E = args.e2e_steps
    sp_h = sp_all[fr:fr + E2E_WARMUP + E2E_WINDOWS * E + 1].cpu().pin_memory()
    vw_h = vw.cpu().pin_memory()
    sp_d = [torch.empty((1, 6), dtype=dt, device=device) for _ in range(2)]
    vw_d = [torch.empty_like(vw) for _ in range(2)]
    h2d = sp_d[0].numel() * sp_d[0].element_size() + vw_d[0].numel() * vw_d[0].element_size()
    copy = torch.cuda.Stream(device)
    import ctypes as C
    hist_d = [fs.alloc_history(1) for _ in range(2)]
    c_hist = [_abi_mod().DemHistory(*[C.c_void_p(int(t.data_ptr())) for t in h]) for h in hist_d]
    io = [(C.c_void_p(int(sp_d[b].data_ptr())), C.c_void_p(int(vw_d[b].data_ptr())), c_hist[b]) for b in range(2)]
    outs_h = [[torch.empty(h.shape, dtype=h.dtype, pin_memory=True) for h in hist_d[0]] for _ in range(2)]
    d2h = sum(h.numel() * h.element_size() for h in hist_d[0])
    torch.cuda.synchronize()
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_done = [torch.cuda.Event() for _ in range(2)]

    def e2e_steps(r0: int, count: int) -> float:
        """`count` steps on setpoint rows r0, r0 + 1, ...; returns their device time [s]."""
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        copy.wait_event(e0)
        with torch.cuda.stream(copy):
            sp_d[0].copy_(sp_h[r0:r0 + 1], non_blocking=True)
            vw_d[0].copy_(vw_h, non_blocking=True)
        ev_in[0].record(copy)
        for i in range(count):
            b = i & 1
            flush.fill_(i & 0xFF)  # evict L2 before every step, as in the device-timed loop
            stream.wait_event(ev_in[b])
            rc_call = direct.frame(0, io[b])
            if rc_call != 0:
                raise RuntimeError(f"dem_scan_segment returned {rc_call}: {fs._error()}")
            ev_done[b].record(stream)
            with torch.cuda.stream(copy):
                if i + 1 < count:
                    # buffer 1-b was last read by step i-1, which the copy stream
                    # already waited for before downloading its results
                    sp_d[1 - b].copy_(sp_h[r0 + i + 1:r0 + i + 2], non_blocking=True)
                    vw_d[1 - b].copy_(vw_h, non_blocking=True)
                    ev_in[1 - b].record(copy)
                copy.wait_event(ev_done[b])
                for hh, hd in zip(outs_h[b], hist_d[b]):
                    hh.copy_(hd, non_blocking=True)
        stream.wait_stream(copy)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3

    e2e_steps(1, E2E_WARMUP)  # the same loop, untimed
    # E2E_WINDOWS consecutive timed windows of E steps; the reported value is
    # their median, so that one host stall (the process descheduled on a shared
    # machine) does not decide the figure; every window is listed
    windows = []
    for wi in range(E2E_WINDOWS):
        if world > 1:
            dist.barrier()
        gc.collect()
        gc.disable()  # no collector pause inside the timed region
        try:
            windows.append(max_over_ranks(e2e_steps(1 + E2E_WARMUP + wi * E, E), world, device))
        finally:
            gc.enable()
    e2e_s = sorted(windows)[len(windows) // 2]
    e2e_value = world * n * N_SUB * E / e2e_s
    rc = fs.lib.dem_sync_status(fs._h, fs._stream())
    if rc != 0:
        raise RuntimeError(f"device status {rc}: {fs._error()}")
    info = fs.info()
    if args.phase_times and args.launch == "persistent":
        print_phase_times(fs, st, sh, sp_all[fr:fr + 1], vw)
        print_phase_times(fs, st, sh, sp_all[fr:fr + 1], vw, flush=flush)

    if rank != 0:
        return None
    bpf = algorithmic_bytes_per_frame(n, nb, V, N_SUB, n_act, nb_act)
    achieved = bpf / frame_s / 1e9
    peak, peak_kind = peak_hbm()
    workload = f"{args.config}{'-allactive' if args.all_active else ''}-seed{args.seed}-{args.dtype}"
    traffic = committed_traffic(workload)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": 1e3 * frame_max, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": args.dtype, "data": "synthetic (seeded field generator)",
        "config": {"workload": f"plain DEM, {args.config} field: {n} elements, {nb} bonds, max_v {V}, "
                               f"{N_SUB} substeps of {DT / N_SUB:g} s per step (frame)",
                   "elements": n, "bonds": nb, "substeps_per_step": N_SUB, "seed": args.seed,
                   "l2": "flushed before every timed step (256 MB write), device-timed and end-to-end loops",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "launch": ("one cooperative persistent kernel per frame" if args.launch == "persistent"
                              else "one kernel launch per phase"),
                   "all_active": bool(args.all_active),
                   "timing": (f"CUDA events around each frame's C-ABI call on the launch stream, host "
                              f"enqueued ahead; value = median of {nwin} consecutive windows' mean frame time"),
                   "frame_windows_ms": [round(x, 5) for x in win_ms],
                   "neighbor_rebuild_rounds": info["neighbor_rebuilds"],
                   "elements_reref_total": info["escaped_total"],
                   "lists_rebuilt_total": info["rebuilt_lists_total"],
                   "max_neighbors": fs.params.max_neighbors, "bucket_capacity": fs.params.bucket_capacity,
                   "skin_m": fs.params.skin,
                   "active_elements": [act0[0], act1[0]], "bonds_with_active_end": [act0[1], act1[1]]},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": f"{peak_kind} copy bandwidth",
                     "algorithmic_bytes_per_launch": bpf,
                     "algorithmic_bytes_if_all_active": algorithmic_bytes_per_frame(n, nb, V, N_SUB),
                     "traffic": traffic},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "steps": E,
                "windows": [world * n * N_SUB * E / w for w in windows],
                "value_of": f"median of {E2E_WINDOWS} consecutive timed windows of {E} steps",
                "path": "pinned host rows -> device, one dem_scan_segment frame through the C ABI, history "
                        "rows -> pinned host, per step"},
        "gpu_launches": K if args.launch == "persistent" else None,
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(field, args.cpu_seconds)
    return line


ROLLOUT_METRIC = "planner rollouts/s"
ROLLOUT_UNIT = "rollouts/s"


def run_rollouts(args, rank: int, world: int):
    """Batched planner rollouts: Q candidates x H control steps on their own ice
    windows cut from the medium field, one persistent launch per batch plus the
    device cost kernel; a step is one batch."""
    import numpy as np
    import torch
    _pkg()
    from mbd_icenav_b200 import rollouts
    device = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(device)
    field = load_field("medium", args.seed)
    dt = torch.float32 if args.dtype == "f32" else torch.float64
    wl = rollouts.planner_workload(field, Q=args.rollouts, H=args.horizon, seed=args.seed + 1000 * rank, dtype=dt,
                                   device=device, bucket_capacity=args.bucket_capacity, skin=args.skin)
    b = wl.batch
    fs = b.frame_step
    Q, H = b.n_rollouts, args.horizon
    n, nb, V = fs.n, fs.n_bonds, fs.max_v
    K, W = args.steps, args.warmup
    stream = torch.cuda.current_stream(device)
    u_d = torch.as_tensor(wl.controls, dtype=dt, device=device)
    vw = torch.zeros((H, n, 2), dtype=dt, device=device)  # still water
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=device)
    cost_out = torch.empty((Q, 5), dtype=torch.float64, device=device)

    def step(u, check=False):
        res = rollouts.run(b, u, vw, history="ship", check=check)
        mid = torch.cuda.Event(enable_timing=True)
        mid.record(stream)
        rollouts.costs(b, res, wl.costmap, wl.goal, wl.ship_length, wl.ship_beam, out=cost_out)
        return res, mid

    for _ in range(W):
        step(u_d, check=True)
    # the work split of this batch shape, picked by timing every choice (all
    # give identical results); untimed
    from mbd_icenav_b200 import autotune
    split, split_ms = autotune.tune(fs, lambda: rollouts.run(b, u_d, vw, history="ship", check=False))
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    mids = [None] * K
    for attempt in range(4):
        with ClockSampler(device.index) as clk:
            torch.cuda.synchronize()
            for i in range(K):
                flush.fill_(i & 0xFF)  # evict L2 before every timed batch
                starts[i].record(stream)
                _, mids[i] = step(u_d)
                ends[i].record(stream)
            torch.cuda.synchronize()
        rc = fs.lib.dem_sync_status(fs._h, fs._stream())
        msg = fs._error() if rc != 0 else ""
        grown = rc == _abi_mod().DEM_ERR_CAPACITY and attempt < 3 and fs.grow_capacity()
        verdict = retry_verdict(rc, grown, world, device)
        if verdict == 0:
            break
        if verdict == 2:
            raise RuntimeError(f"device status {rc}: {msg}" if rc else "device error on another rank")
    res_end, _ = step(u_d)
    bi, bj = fs._keep["bi"], fs._keep["bj"]
    act0 = active_counts(b.state.elem_active, bi, bj)
    act1 = active_counts(res_end.state.elem_active, bi, bj)
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    kern_ms = [s.elapsed_time(m) for s, m in zip(starts, mids)]
    total_s = sum(step_ms) / 1e3
    total_max = max_over_ranks(total_s, world, device)
    value = world * Q * K / total_max

    # end to end through the public API: per batch the controls go up from
    # pinned host memory and the (Q, 5) costs come back, inside the timed region
    E = max(1, min(K, 5))
    u_h = torch.as_tensor(wl.controls, dtype=dt).pin_memory()
    c_h = torch.empty((Q, 5), dtype=torch.float64, pin_memory=True)
    u_in = torch.empty_like(u_d)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    gc.collect()
    gc.disable()  # no collector pause inside the timed region
    try:
        e0.record(stream)
        for i in range(E):
            flush.fill_(i & 0xFF)  # evict L2 before every batch, as in the device-timed loop
            u_in.copy_(u_h, non_blocking=True)
            step(u_in)
            c_h.copy_(cost_out, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
    finally:
        gc.enable()
    e2e_value = world * Q * E / max_over_ranks(e0.elapsed_time(e1) / 1e3, world, device)
    rc = fs.lib.dem_sync_status(fs._h, fs._stream())
    if rc != 0:
        raise RuntimeError(f"device status {rc}: {fs._error()}")
    c = c_h.numpy()
    if not np.isfinite(c).all():
        raise RuntimeError("non-finite rollout costs")
    info = fs.info()
    if args.phase_times:
        print_phase_times(fs, None, None, None, None, frames=1, frames_per_run=H,
                          run=lambda: rollouts.run(b, u_d, vw, history="ship", check=False))
    if rank != 0:
        return None
    sizes = np.diff(b.system_start)
    # the batch's first frame carries frozen elements over; the other H - 1
    # frames update the state in place
    na_m, nba_m = 0.5 * (act0[0] + act1[0]), 0.5 * (act0[1] + act1[1])
    bpl = (algorithmic_bytes_per_frame(n, nb, V, N_SUB, act0[0], act0[1])
           + (H - 1) * algorithmic_bytes_per_frame(n, nb, V, N_SUB, na_m, nba_m, in_place=True))
    kern_s = sum(kern_ms) / 1e3 / K
    achieved = bpl / kern_s / 1e9
    peak, peak_kind = peak_hbm()
    line = {
        "metric": ROLLOUT_METRIC, "value": value, "unit": ROLLOUT_UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": 1e3 * total_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": args.dtype, "data": "synthetic (seeded medium field, seeded Gaussian controls)",
        "config": {"workload": f"batched planner rollouts: {Q} candidates x {H} control steps x {N_SUB} substeps, "
                               f"windows of {int(sizes.min())}-{int(sizes.max())} elements (mean "
                               f"{sizes.mean():.0f}) cut from the medium field along each path, "
                               f"{wl.costmap.rows}x{wl.costmap.cols} costmap of 2 m cells + transferred ice KE",
                   "rollouts": Q, "horizon": H, "elements": n, "bonds": nb, "seed": args.seed,
                   "step_ms": [round(x, 3) for x in step_ms],
                   "elem_steps_per_s": value * sizes.mean() * H * N_SUB,
                   "l2": "flushed before every timed batch (256 MB write), device-timed and end-to-end loops",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "launch": "one cooperative persistent kernel per batch (all H steps) + one cost kernel",
                   "neighbor_rebuild_rounds": info["neighbor_rebuilds"],
                   "elements_reref_total": info["escaped_total"],
                   "lists_rebuilt_total": info["rebuilt_lists_total"],
                   "max_neighbors": fs.params.max_neighbors, "bucket_capacity": fs.params.bucket_capacity,
                   "skin_m": fs.params.skin,
                   "active_elements": [act0[0], act1[0]], "bonds_with_active_end": [act0[1], act1[1]],
                   "work_split": split, "work_split_ms": split_ms,
                   "mean_transferred_ke_J": float(c[:, 4].mean()),
                   "rollouts_touching_ice": int((c[:, 4] > 0).sum())},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": f"{peak_kind} copy bandwidth", "algorithmic_bytes_per_launch": bpl,
                     "algorithmic_bytes_if_all_active": H * algorithmic_bytes_per_frame(n, nb, V, N_SUB),
                     "kernel_ms_per_launch": 1e3 * kern_s,
                     "traffic": committed_traffic(f"rollouts-Q{Q}-H{H}-seed{args.seed}-{args.dtype}")},
        "e2e": {"value": e2e_value, "unit": ROLLOUT_UNIT, "h2d_bytes_per_step": int(u_h.numel() * u_h.element_size()),
                "d2h_bytes_per_step": int(c_h.numel() * c_h.element_size()), "steps": E},
        "gpu_launches": 2 * K,
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu_baseline:
        m = int(round(sizes.mean()))
        steps, secs, frames, nw = _oracle_frames(field, field.trajectory[START_FRAME], m, args.cpu_seconds,
                                                 min_frames=2)
        line["cpu_baseline"] = {"value": frames / secs / H, "unit": ROLLOUT_UNIT, "cores": 1, "kind": "port",
                                "sample": f"NumPy oracle (float64), {frames} frames x {N_SUB} substeps on one "
                                          f"{nw}-element window (the batch's mean window size) of the same field; "
                                          f"rollouts/s = frames/s / {H} steps; one core"}
    return line


SUR_METRIC = "MBD candidates scored/s (surrogate-screened)"
SUR_UNIT = "rollouts/s"


def run_surrogate(args, rank: int, world: int):
    """Surrogate-screened MBD planning against the plain batched-DEM MBD: the
    network is trained (untimed) on DEM rollouts of the medium field, then both
    planners plan from held-out starts; a step is one plan (n_diffuse - 1
    reverse steps of n_sample candidates).  value = candidates scored per
    second by the screened planner; the plain planner's rate and the relative
    difference of the two plans' DEM costs are reported beside it."""
    import numpy as np
    import torch
    _pkg()
    from mbd_icenav_b200 import planner, sg_ops, surrogate as S
    device = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(device)
    field = load_field("medium", args.seed)
    H = args.horizon
    t0 = time.time()
    data = planner.generate_dataset(field, n_starts=args.sur_starts, per_start=args.sur_per_start, horizon=H,
                                    seed=args.seed + 100 * rank, device=device, scenes=args.sur_scenes)
    gen_s = time.time() - t0
    rank_corr = planner.within_scene_rank_corr(data)
    sur, info = planner.train_surrogate(data, horizon=H, epochs=args.sur_epochs, batch=256, device=device,
                                        seed=args.seed)
    cfg = planner.MBDConfig(horizon=H, n_sample=args.sur_samples, n_diffuse=args.sur_iters + 1,
                            top_k=args.sur_top_k)
    w = planner.CostWeights()
    rng = np.random.default_rng(args.seed + 7777)
    starts = planner.scene_starts(field, args.sur_scenes, args.steps + args.warmup, rng, H)
    stream = torch.cuda.current_stream(device)

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return out, e0.elapsed_time(e1) / 1e3

    rows = []
    with ClockSampler(device.index) as clk:
        for si, (e0, rem) in enumerate(starts):
            sc = planner.make_scene(field, e0, (2.0, 0.0, 0.0), H, device=device, patch_stats=data.patch_stats,
                                    removed=rem)
            plain = planner.DemScorer(sc, cfg.n_sample, w)
            scr = planner.ScreenedScorer(sc, sur, cfg.n_sample, w, top_k=cfg.top_k, max_rel_err=cfg.max_rel_err,
                                         n_check=args.sur_check, seed=si, adapt_steps=args.sur_adapt)
            # the configuration's own top-64, for comparison
            scr64 = planner.ScreenedScorer(sc, sur, cfg.n_sample, w, top_k=64, max_rel_err=cfg.max_rel_err,
                                           n_check=args.sur_check, seed=si, adapt_steps=args.sur_adapt)
            # the same screening with the network learning the scene as the plan goes
            scra = planner.ScreenedScorer(sc, sur, cfg.n_sample, w, top_k=cfg.top_k, max_rel_err=cfg.max_rel_err,
                                          n_check=args.sur_check, seed=si, adapt_steps=args.sur_compare_adapt)
            # the same screening with a band below the top-k checked, and scored in full on a miss
            scrd = planner.ScreenedScorer(sc, sur, cfg.n_sample, w, top_k=cfg.top_k, max_rel_err=cfg.max_rel_err,
                                          n_check=args.sur_check, seed=si, adapt_steps=args.sur_adapt,
                                          deepen=args.sur_deepen)
            # untimed: each DEM batch's work split, tuned on candidates like a plan's
            Yt = torch.clamp(torch.randn((cfg.n_sample, H, 2), device=device) * 0.3 + 0.7, -1, 1)
            split_plain, _ = plain.autotune(Yt)
            split_k, _ = scr.dem_k.autotune(Yt[:scr.dem_k.Q].contiguous())
            scr64.dem_k.autotune(Yt[:scr64.dem_k.Q].contiguous())
            scra.dem_k.autotune(Yt[:scra.dem_k.Q].contiguous())
            scrd.dem_k.autotune(Yt[:scrd.dem_k.Q].contiguous())
            (Yp, _), tp = timed(lambda: planner.mbd_plan(plain, cfg, device, seed=si))
            n_fb0 = scr.fallbacks
            (Ys, _), ts = timed(lambda: planner.mbd_plan(scr, cfg, device, seed=si))
            scr.restore()  # each plan starts from the trained network
            (Ys64, _), ts64 = timed(lambda: planner.mbd_plan(scr64, cfg, device, seed=si))
            scr64.restore()
            (Ysa, _), tsa = timed(lambda: planner.mbd_plan(scra, cfg, device, seed=si))
            scra.restore()
            (Ysd, _), tsd = timed(lambda: planner.mbd_plan(scrd, cfg, device, seed=si))
            scrd.restore()
            # the plain planner again with other samples: its own spread of plan costs
            Yp2, _ = planner.mbd_plan(plain, cfg, device, seed=si + 1000)
            cp = planner.plan_cost(sc, Yp, scr.dem_k)
            cs = planner.plan_cost(sc, Ys, scr.dem_k)
            cp2 = planner.plan_cost(sc, Yp2, scr.dem_k)
            cs64 = planner.plan_cost(sc, Ys64, scr.dem_k)
            csa = planner.plan_cost(sc, Ysa, scr.dem_k)
            csd = planner.plan_cost(sc, Ysd, scr.dem_k)
            if si >= args.warmup:
                rows.append({"plain_s": tp, "screened_s": ts, "plain_cost": cp, "screened_cost": cs,
                             "plain_cost_other_seed": cp2,
                             "rel_cost_err": abs(cs - cp) / max(abs(cp), 1e-9),
                             "plain_seed_spread": abs(cp2 - cp) / max(abs(cp), 1e-9),
                             "fallbacks": scr.fallbacks - n_fb0,
                             "check_miss_max": float(np.max(scr.rel_errs)),
                             "pred_rel_err_mean": float(np.mean(scr.pred_errs)), "window": int(len(sc.window)),
                             "work_split": [split_plain, split_k],
                             "top64": {"screened_s": ts64, "screened_cost": cs64,
                                       "rel_cost_err": abs(cs64 - cp) / max(abs(cp), 1e-9),
                                       "fallbacks": scr64.fallbacks, "check_miss_max": float(np.max(scr64.rel_errs))},
                             "adaptive": {"screened_s": tsa, "screened_cost": csa,
                                          "rel_cost_err": abs(csa - cp) / max(abs(cp), 1e-9),
                                          "fallbacks": scra.fallbacks,
                                          "check_miss_max": float(np.max(scra.rel_errs))},
                             "deepen": {"screened_s": tsd, "screened_cost": csd,
                                        "rel_cost_err": abs(csd - cp) / max(abs(cp), 1e-9),
                                        "fallbacks": scrd.fallbacks, "deepened": scrd.deepened,
                                        "band_miss_max": float(np.max(scrd.band_errs)),
                                        "check_miss_max": float(np.max(scrd.rel_errs))}})
                sys.stderr.write(f"plan {si}: {json.dumps(rows[-1])}\n")
            plain.batch.frame_step.close()
            for z in (scr, scr64, scra, scrd):
                z.close()
            del plain, scr, scr64, scra, scrd
    # tensor-pipe figure: the screening's own network work on one plan's
    # population, the head over n_sample rows after one encoder pass, timed alone
    sc = planner.make_scene(field, starts[-1][0], (2.0, 0.0, 0.0), H, device=device, patch_stats=data.patch_stats,
                            removed=starts[-1][1])
    Yn = torch.clamp(torch.randn((cfg.n_sample, H, 2), device=device) * 0.3 + 0.5, -1, 1)
    ext = planner.features(sc, Yn, *planner.rigid_path(sc, Yn)[1:])
    rows0 = torch.zeros(cfg.n_sample, dtype=torch.int32, device=device)
    enc = sur.net.encode(sc.patch, tag="bench_enc")
    for _ in range(3):
        sur.net.head(enc, ext, enc_row=rows0, tag="bench_head")
    _, t_fwd = timed(lambda: [sur.net.head(enc, ext, enc_row=rows0, tag="bench_head") for _ in range(20)])
    fl = S.flops_per_sample(H)
    tflops = 20 * cfg.n_sample * fl["mlp"] / t_fwd / 1e12
    sg_ops.error_flag(device).check()
    if rank != 0:
        return None
    K = len(rows)
    cand = cfg.n_sample * cfg.n_diffuse - cfg.n_sample  # candidates scored per plan
    ts = sum(r["screened_s"] for r in rows) / K
    tp = sum(r["plain_s"] for r in rows) / K
    ts_max = max_over_ranks(ts, world, device)
    tp_max = max_over_ranks(tp, world, device)
    value = world * cand / ts_max
    plain_rate = world * cand / tp_max
    errs = [r["rel_cost_err"] for r in rows]
    peak_tf = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peak_tf = float(json.load(fh)["bf16_tflops"])
        peak_kind = "measured"
    except Exception:
        peak_tf, peak_kind = 1590.0, "fallback"
    line = {
        "metric": SUR_METRIC, "value": value, "unit": SUR_UNIT, "n_gpus": world, "steps": K, "warmup": args.warmup,
        "ms_per_step": 1e3 * ts_max, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 DEM, bf16 surrogate (fp32 accumulate)",
        "data": f"synthetic (seeded medium field, {args.sur_scenes} starts; training tuples from the DEM's own "
                "batched rollouts)",
        "config": {"workload": f"MBD {cfg.n_sample} samples x {cfg.n_diffuse - 1} reverse steps, horizon {H} x "
                               f"10 substeps, top {cfg.top_k} + {args.sur_check} random re-scored by the DEM, "
                               f"fallback when the random ones beat the screened best by {cfg.max_rel_err:.0%}, "
                               f"{args.sur_adapt} Adam steps per MBD step on the check set",
                   "top64": {"speedup_vs_plain_dem": tp / (sum(r["top64"]["screened_s"] for r in rows) / K),
                             "plan_rel_cost_err": [r["top64"]["rel_cost_err"] for r in rows],
                             "fallback_steps": [r["top64"]["fallbacks"] for r in rows],
                             "note": "the same plans with only the 64 best-ranked candidates re-scored"},
                   "adaptive": {"speedup_vs_plain_dem": tp / (sum(r["adaptive"]["screened_s"] for r in rows) / K),
                                "plan_rel_cost_err": [r["adaptive"]["rel_cost_err"] for r in rows],
                                "fallback_steps": [r["adaptive"]["fallbacks"] for r in rows],
                                "note": f"the same plans with {args.sur_compare_adapt} Adam steps per MBD step on "
                                        f"the check set (every candidate after a fallback)"},
                   "deepen": {"speedup_vs_plain_dem": tp / (sum(r["deepen"]["screened_s"] for r in rows) / K),
                              "plan_rel_cost_err": [r["deepen"]["rel_cost_err"] for r in rows],
                              "fallback_steps": [r["deepen"]["fallbacks"] for r in rows],
                              "deepened_steps": [r["deepen"]["deepened"] for r in rows],
                              "note": f"the same plans with half the check drawn from the {args.sur_deepen} "
                                      f"candidates ranked below the top {cfg.top_k}, all of which the DEM scores "
                                      f"when that half beats the screened best"},
                   "scenes": args.sur_scenes, "windows": [r["window"] for r in rows],
                   "plain_dem_rollouts_per_s": plain_rate, "speedup_vs_plain_dem": value / plain_rate,
                   "plan_rel_cost_err": errs, "plan_rel_cost_err_max": max(errs),
                   "plans_within_5pct": int(sum(e <= 0.05 for e in errs)),
                   "plain_seed_spread": [r["plain_seed_spread"] for r in rows], "plans": rows,
                   "train": {"samples": info["train_samples"], "holdout_samples": info["holdout_samples"],
                             "epochs": args.sur_epochs, "steps": info["steps"], "seconds": info["seconds"],
                             "holdout_mse_std_units": info["holdout_loss"], "train_loss": info["train_loss"],
                             "data_seconds": gen_s, "starts": args.sur_starts, "per_start": args.sur_per_start,
                             "within_scene_rank_corr": rank_corr},
                   "network": {"params": sur.net.n_params(), "flops_per_sample_fwd": fl},
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "roofline": {"bound": "tensor", "achieved": tflops, "peak": peak_tf, "unit": "TFLOP/s",
                     "frac": tflops / peak_tf, "peak_kind": f"{peak_kind} bf16 dense",
                     "what": f"surrogate head (3 x 512 MLP + output, bf16 tcgen05 GEMMs) on {cfg.n_sample} rows "
                             f"after one encoder pass: the screening's network work per MBD step, 20 passes timed",
                     "traffic": None},
        "e2e": {"value": value, "unit": SUR_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 8,
                "note": "plans read their controls from device buffers; the plan's cost comes back"},
        "gpu_launches": None,
        "clocks": clk.summary(),
    }
    return line


def print_phase_times(fs, st, sh, sp, vw, frames: int = 5, run=None, frames_per_run: int = 1, flush=None):
    """Per-phase device time of a few frames (profiling switch of the library).
    ``run()`` replaces the default one-frame scan (``frames`` calls of it, each
    ``frames_per_run`` frames long); ``flush``, a buffer larger than L2, is
    written before every call."""
    import collections
    import torch
    k = fs.n_ice_steps
    per = 5 + 3 * k
    names = ["cull", "near", "cforce", "reduce"] + [f"{x}" for s in range(k)
                                                     for x in ("escape", "build_all", "force")] + ["fracture"]
    acc = collections.defaultdict(list)
    per_sub = collections.defaultdict(list)
    fs.set_profiling(True)
    for i in range(frames):
        if flush is not None:
            flush.fill_(i & 0xFF)
        if run is None:
            st, sh, _ = fs.scan_segment(st, sh, sp, vw, history=False)
        else:
            run()
        torch.cuda.synchronize()
        pts = fs.phase_times()
        prev = 0
        for ph, t in pts:
            acc[names[ph % per]].append((t - prev) / 1e3)
            p = ph % per
            if 4 <= p < per - 1:
                per_sub[(names[p], (p - 4) // 3)].append((t - prev) / 1e3)
            prev = t
    fs.set_profiling(False)
    tot = 0.0
    frames = frames * frames_per_run
    for nm in ("cull", "near", "cforce", "reduce", "escape", "build_all", "force", "fracture"):
        v = acc.get(nm, [])
        s = sum(v) / frames
        tot += s
        sys.stderr.write(f"phase {nm:9s} {s:9.1f} us/frame  ({len(v) / frames:.1f} runs/frame)\n")
    sys.stderr.write(f"phase total     {tot:9.1f} us/frame{' (L2 flushed before each call)' if flush is not None else ''}\n")
    for nm in ("escape", "force"):
        row = " ".join(f"{sum(per_sub[(nm, i)]) / max(len(per_sub[(nm, i)]), 1):6.1f}" for i in range(k))
        sys.stderr.write(f"phase {nm:9s} by substep (us per run): {row}\n")


# ── CPU side (the oracle is the checker/baseline only) ─────────────────────────

def _window(field, center, n_keep, keep=None):
    """The n_keep elements nearest ``center`` (or the elements ``keep``) as a
    field of their own: bonds and floes inside it only."""
    import numpy as np
    if keep is None:
        d = np.linalg.norm(field.centroids - np.asarray(center)[None, :2], axis=1)
        keep = np.argsort(d)[:n_keep]
    keep = np.sort(np.asarray(keep, np.int64))
    remap = -np.ones(field.n, np.int64)
    remap[keep] = np.arange(len(keep))
    bonds = [(int(remap[i]), int(remap[j])) for i, j in field.bonds if remap[i] >= 0 and remap[j] >= 0]
    _, parents = np.unique(field.parent_ids[keep], return_inverse=True)
    return [field.polygons[k] for k in keep], field.centroids[keep], bonds, field.thicknesses[keep], parents


def _oracle_for(field, window):
    import numpy as np
    from mbd_icenav_b200.config import SimulationConfig
    from mbd_icenav_b200.state import build_static_arrays, initial_ice_state_arrays, ship_dynamics_arrays
    from mbd_icenav_b200.vessel import SupplyVessel
    from oracle.dem_oracle import OShip, OState, Oracle, params_from_config
    polys, cents, bonds, thick, parents = window
    cfg = SimulationConfig()
    sa = build_static_arrays(polys, cents, bonds, thick, parents, cfg, dilation=0.05)
    sd = ship_dynamics_arrays(field.ship_props, cfg, field.ship_length, field.ship_beam, field.hull_local)
    sv = SupplyVessel(mass=field.ship_props.mass, length=field.ship_length)
    o = Oracle(sa, sd, params_from_config(cfg, field.ship_length, field.ship_beam, N_SUB, DT, DT / N_SUB,
                                          False, sv.T_n), sv.B, np.float64, pair_mode="grid")
    st = OState(*initial_ice_state_arrays(len(polys), cents, len(bonds), parents))
    return o, st, OShip


def _oracle_frames(field, center, n_keep, seconds, min_frames=1, max_frames=10 ** 9, keep=None):
    """Run oracle frames on a window until `seconds` elapse; return (element-steps, seconds)."""
    import numpy as np
    o, st, OShip = _oracle_for(field, _window(field, center, n_keep, keep))
    eta0 = field.trajectory[START_FRAME]
    sh = OShip(np.array(eta0, float), np.zeros(3), np.zeros(6), np.zeros(3))
    n = o.n
    vw = np.tile(np.asarray(field.current, float), (n, 1))
    sp = field.setpoints(START_FRAME, max(min_frames, 1) + 10000)
    t0 = time.perf_counter()
    frames = 0
    while frames < max_frames and (frames < min_frames or time.perf_counter() - t0 < seconds):
        st, sh, _ = o.frame_step(st, sh, sp[frames % len(sp), :3], sp[frames % len(sp), 3:], vw,
                                 st.dpdem_floe_eligible)
        frames += 1
    return n * N_SUB * frames, time.perf_counter() - t0, frames, n


def cpu_baseline(field, seconds: float):
    steps, secs, frames, n = _oracle_frames(field, field.trajectory[START_FRAME], 16384, seconds, min_frames=2)
    return {"value": steps / secs, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"NumPy oracle (float64, restated broad phase), {frames} frames x {N_SUB} substeps "
                      f"on a {n}-element window of the same field around the ship; NumPy runs on one core"}


def _ref_worker(argv):
    name, seed, center, n_keep, seconds, frames = argv[:6]
    slab = argv[6] if len(argv) > 6 else None  # (index, count): a slab of the field by x
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "mbd-icenav_b200"))
    _pkg()
    field = load_field(name, seed)
    keep = None
    if slab is not None:
        import numpy as np
        keep = np.array_split(np.argsort(field.centroids[:, 0], kind="stable"), slab[1])[slab[0]]
    return _oracle_frames(field, center, n_keep, seconds, min_frames=frames, max_frames=frames, keep=keep)


def field_slabs(n: int, procs: int):
    """Element counts of the field's ``procs`` slabs by x (``_ref_worker``)."""
    import numpy as np
    return [len(a) for a in np.array_split(np.arange(n), procs)]


def run_reference(args):
    """Oracle port on all host cores: one process per core, each on its own window."""
    import multiprocessing as mp
    import numpy as np
    _pkg()
    if args.config in ("rollouts", "surrogate"):
        # the CPU reference rate of scoring candidates: the oracle port rolling
        # candidates out on the host cores (the reference has no surrogate)
        return run_reference_rollouts(args)
    field = load_field(args.config, args.seed)
    cores = len(os.sched_getaffinity(0))
    procs = max(1, min(cores, 32))
    K, W = args.steps, args.warmup
    # the whole field, split into one slab (by x) per process, so that every
    # element of the bench's field is stepped each frame; the port computes
    # every element, active or frozen, as the reference's algorithm does
    per_proc = max(field_slabs(field.n, procs))
    # ~2.5e5 element-steps/s per core for the port (measured): frames per process
    # so that the timed part stays within ~240 s
    frames = int(max(1, min(K, 240.0 * 2.5e5 / (per_proc * N_SUB))))
    ctr = field.trajectory[START_FRAME]
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        jobs = [(args.config, args.seed, ctr, 0, 0.0, 1, (i, procs)) for i in range(procs)]
        pool.map(_ref_worker, jobs)  # warm-up: field load + one frame per worker
        t0 = time.perf_counter()
        res = pool.map(_ref_worker, [(args.config, args.seed, ctr, 0, 0.0, frames, (i, procs))
                                     for i in range(procs)])
        wall = time.perf_counter() - t0
    steps = sum(r[0] for r in res)
    value = steps / wall
    n_all = sum(r[3] for r in res)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0,
            "steps": frames, "warmup": W, "ms_per_step": 1e3 * wall / frames, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded field generator)",
            "config": {"workload": f"plain DEM, {args.config} field: all {n_all} elements as {procs} slabs "
                                   f"by x, one per process, NumPy oracle port",
                       "elements": n_all, "processes": procs, "frames": frames,
                       "elements_per_process": [r[3] for r in res]},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": "port",
                             "sample": f"{frames} frames x {N_SUB} substeps of the whole field ({n_all} "
                                       f"elements) as {procs} independent slabs (restated broad phase; "
                                       f"bonds and contacts across slab borders left out); the reference "
                                       f"JAX code cannot be installed in this image"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    return line


def run_reference_rollouts(args):
    """Oracle port on all host cores for the rollout workload: each process rolls
    out one candidate per step (H frames) on its own window of the medium field,
    of the batch's mean window size."""
    import multiprocessing as mp
    import numpy as np
    K, W, H = args.steps, args.warmup, args.horizon
    field = load_field("medium", args.seed)
    cores = len(os.sched_getaffinity(0))
    procs = max(1, min(cores, 32))
    n_keep = 1011  # mean window of the 2048-candidate batch (log-uniform 200-3000 elements)
    rng = np.random.default_rng(args.seed)
    near = np.argsort(np.linalg.norm(field.centroids - field.trajectory[START_FRAME][:2], axis=1))[:procs * 8]
    centers = field.centroids[rng.choice(near, procs, replace=False)]
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        pool.map(_ref_worker, [("medium", args.seed, c, n_keep, 0.0, 1) for c in centers])  # warm-up
        t0 = time.perf_counter()
        res = pool.map(_ref_worker, [("medium", args.seed, c, n_keep, 0.0, H * K) for c in centers])
        wall = time.perf_counter() - t0
    rollouts_done = procs * K
    value = rollouts_done / wall
    sample = (f"{K} rollouts x {H} frames x {N_SUB} substeps per process on {procs} windows of "
              f"{res[0][3]} elements near the ship (restated broad phase); the reference JAX code cannot be "
              f"installed in this image")
    return {"impl": "reference", "metric": ROLLOUT_METRIC, "value": value, "unit": ROLLOUT_UNIT, "n_gpus": 0,
            "steps": K, "warmup": W, "ms_per_step": 1e3 * wall / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded medium field)",
            "config": {"workload": f"planner rollouts, NumPy oracle port: {procs} processes, one candidate of "
                                   f"{H} steps each per step", "processes": procs, "horizon": H,
                       "elements_per_window": n_keep},
            "cpu_baseline": {"value": value, "unit": ROLLOUT_UNIT, "cores": procs, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": ROLLOUT_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=["large", "medium", "small", "rollouts", "surrogate"], default="large",
                    help="plain-DEM field, or batched planner rollouts on windows of the medium field")
    ap.add_argument("--rollouts", type=int, default=2048, help="candidates per batch (--config rollouts)")
    ap.add_argument("--horizon", type=int, default=64, help="control steps per candidate (--config rollouts)")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--dtype", choices=["f32", "f64"], default="f32")
    ap.add_argument("--e2e-steps", type=int, default=200)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--launch", choices=["persistent", "phased"], default="persistent")
    ap.add_argument("--skin", type=float, default=0.8, help="Verlet skin of the neighbour lists [m]")
    ap.add_argument("--bucket-capacity", type=int, default=64,
                    help="grid-bucket capacity at start (grown automatically on overflow)")
    ap.add_argument("--order", choices=["floe", "morton"], default="floe",
                    help="element numbering: as generated (by floe) or Morton order of centroids")
    ap.add_argument("--phase-times", action="store_true",
                    help="after the run, time one profiled frame per phase (device clock) to stderr")
    ap.add_argument("--sur-starts", type=int, default=1024, help="training starts (--config surrogate)")
    ap.add_argument("--sur-per-start", type=int, default=256, help="DEM rollouts per training start")
    ap.add_argument("--sur-epochs", type=int, default=10)
    ap.add_argument("--sur-samples", type=int, default=8192, help="MBD samples per reverse step")
    ap.add_argument("--sur-iters", type=int, default=16, help="MBD reverse steps per plan")
    ap.add_argument("--sur-top-k", type=int, default=512, help="best-ranked candidates re-scored by the DEM per step")
    ap.add_argument("--sur-check", type=int, default=64, help="random held-out candidates re-scored per step")
    ap.add_argument("--sur-adapt", type=int, default=0,
                    help="Adam steps per MBD step on the check set the DEM scored (0: the network stays fixed)")
    ap.add_argument("--sur-compare-adapt", type=int, default=4,
                    help="Adam steps per MBD step of the adaptive comparison plans")
    ap.add_argument("--sur-deepen", type=int, default=1536,
                    help="band below the top-k for the deepening comparison plans (ScreenedScorer deepen)")
    ap.add_argument("--sur-scenes", choices=("channel", "open"), default="channel",
                    help="plan starts: mid-transit in the pack with the ship's channel cleared, or open water")
    ap.add_argument("--all-active", action="store_true",
                    help="every element active from the start (the force path on the whole field)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank, world, relaunch = resolve_world(args.gpus, os.environ)
    if relaunch:
        return subprocess.call(torchrun_command(args.gpus, _free_port(), sys.argv[1:]))
    if args.impl == "reference":
        if rank != 0:
            return 0
        print(json.dumps(run_reference(args)), flush=True)
        return 0
    body = {"rollouts": run_rollouts, "surrogate": run_surrogate}.get(args.config, run_ours)
    run_ranked(lambda r, w: body(args, r, w), rank, world, backend="nccl")
    return 0


def resolve_world(gpus: int, env) -> tuple:
    """(rank, world size, relaunch) for ``--gpus N``.  Under torchrun the world
    size comes from WORLD_SIZE and must equal N; run without torchrun and with
    N > 1, the bench relaunches itself under torchrun with N ranks."""
    if gpus < 1:
        raise SystemExit("--gpus must be at least 1")
    if "WORLD_SIZE" not in env:
        return 0, 1, gpus > 1
    world = int(env["WORLD_SIZE"])
    if world != gpus:
        raise SystemExit(f"--gpus {gpus} but WORLD_SIZE={world}: one rank per GPU is expected")
    return int(env.get("RANK", 0)), world, False


def torchrun_command(gpus: int, port: int, argv) -> list:
    """The single-node torchrun command that runs this file with one rank per GPU."""
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={gpus}",
            "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__), *argv]


def _free_port() -> int:
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def run_ranked(body, rank: int, world: int, backend: str = "nccl", out=sys.stdout):
    """The rank entry: with world > 1, join the process group (``backend``; one
    CUDA device per rank for nccl), run ``body(rank, world)`` (every rank times
    its replica; the slowest rank's time is taken inside) and print rank 0's
    JSON line; the group is left on every path."""
    if world > 1:
        import datetime
        import torch.distributed as dist
        if backend == "nccl":
            import torch
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    try:
        line = body(rank, world)
        if rank == 0 and line is not None:
            out.write(json.dumps(line) + "\n")
            out.flush()
        return line
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
