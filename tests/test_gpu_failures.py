"""Failure detection on the GPU without a GPU fault.

* A grid barrier that can never complete (one CTA leaves through the test
  hook dem_debug_fail_barrier) ends every other CTA's wait at its 2 s limit:
  the call reports DEM_ERR_TIMEOUT through dem_sync_status, the launch ends by
  itself, and the next call on the same handle is correct.
* NaN injected on the host into the input state goes through the reference's
  sanitisation (jax_simulation.py:239-254): the GPU frame matches the oracle's,
  NaNs included.
"""
import time

import numpy as np
import pytest

from helpers import frame_inputs, gpu_frame_step, initial_state, make_oracle, rel_err, to_gpu_state, to_np_state

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _frame(fs, st, sh, g, prefix, f, dtype, check=True):
    sp, spn, vw, vws = frame_inputs(g, prefix, f)
    d = torch.device("cuda", 0)
    t = lambda a: torch.as_tensor(np.asarray(a, np.float64)).to(d, dtype)
    return fs(st, sh, t(sp), t(spn), t(vw), st.dpdem_floe_eligible, t(vws), check=check)


def test_barrier_timeout_is_reported_and_the_handle_recovers(golden32):
    from mbd_icenav_b200 import _abi
    g = golden32
    prefix = "window"
    o_st, o_sh = initial_state(g, prefix, np.float32)
    fs = gpu_frame_step(g, prefix, torch.float32)
    lib = fs.lib
    assert lib.dem_debug_fail_barrier(fs._h, 2) == _abi.DEM_OK  # after the contact-force phase
    st, sh = to_gpu_state(o_st, o_sh, torch.float32)
    t0 = time.monotonic()
    _frame(fs, st, sh, g, prefix, 0, torch.float32, check=False)
    rc = lib.dem_sync_status(fs._h, fs._stream())
    elapsed = time.monotonic() - t0
    assert rc == _abi.DEM_ERR_TIMEOUT, rc
    assert elapsed < 30.0  # each CTA gave up at its own 2 s limit
    # the same handle, next call: identical to a fresh handle's frame
    st, sh = to_gpu_state(o_st, o_sh, torch.float32)
    a_st, a_sh, _ = _frame(fs, st, sh, g, prefix, 0, torch.float32)
    fresh = gpu_frame_step(g, prefix, torch.float32)
    st, sh = to_gpu_state(o_st, o_sh, torch.float32)
    b_st, b_sh, _ = _frame(fresh, st, sh, g, prefix, 0, torch.float32)
    for a, b in zip(a_st + a_sh, b_st + b_sh):
        assert torch.equal(a, b)
    fs.close()
    fresh.close()


def test_barrier_fault_hook_is_refused_in_phased_mode(golden32):
    from mbd_icenav_b200 import _abi
    fs = gpu_frame_step(golden32, "window", torch.float32)
    fs.set_launch_mode(_abi.DEM_LAUNCH_PHASED)
    assert fs.lib.dem_debug_fail_barrier(fs._h, 2) == _abi.DEM_ERR_INVALID
    fs.close()


def test_nan_inputs_are_sanitised_like_the_reference(golden64):
    g = golden64
    prefix = "window"
    o_st, o_sh = initial_state(g, prefix, np.float64)
    pos = o_st.positions.copy()
    vel = o_st.velocities.copy()
    pos[7] = np.nan         # a position: no contacts, NaN bond forces on its partners
    vel[100, 0] = np.nan    # a velocity: NaN drag and friction, reset to 0 by the update
    o_st = o_st._replace(positions=pos, velocities=vel)
    o = make_oracle(g, prefix, np.float64, pair_mode="all")
    sp, spn, vw, vws = frame_inputs(g, prefix, 0)
    w_st, w_sh, _ = o.frame_step(o_st, o_sh, sp, spn, vw, o_st.dpdem_floe_eligible, vws)
    fs = gpu_frame_step(g, prefix, torch.float64)
    st, sh = to_gpu_state(o_st, o_sh, torch.float64)
    r_st, r_sh, _ = _frame(fs, st, sh, g, prefix, 0, torch.float64)
    ice, ship = to_np_state(r_st, r_sh)
    for name in ("positions", "velocities", "rotations", "angular_vels", "submergence"):
        got, want = getattr(ice, name), getattr(w_st, name)
        np.testing.assert_array_equal(np.isnan(got), np.isnan(want), err_msg=name)
        ok = ~np.isnan(want)
        assert rel_err(got[ok], want[ok], 1e-6) < 1e-9, name
    for name in ("bond_intact", "elem_active", "dpdem_floe_eligible"):
        np.testing.assert_array_equal(getattr(ice, name), getattr(w_st, name), err_msg=name)
    # the reference sanitises ice values only: a NaN that reaches the ship-force
    # sum reaches the vessel state too, on both sides alike
    for name in ("eta", "nu", "n_actual", "e_int"):
        got, want = getattr(ship, name), getattr(w_sh, name)
        np.testing.assert_array_equal(np.isnan(got), np.isnan(want), err_msg=name)
        ok = ~np.isnan(want)
        assert rel_err(got[ok], want[ok]) < 1e-9, name
    fs.close()
