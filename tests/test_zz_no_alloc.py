"""dem_ship_contact_noalloc (the allocation-free contact test) against dem_frame_step.

Both entry points are called through the C ABI on the same input state; the
new one must give the penetration depths that dem_frame_step reports as
diag.pen_max, on two calls in a row (a 500-element float32 window, then a
24-element float64 field), so that the second call runs on scratch the first
one left behind.  This file is collected last and builds everything it needs,
so it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import (frame_inputs, gpu_frame_step, initial_state, make_oracle, rel_err, shipdyn_from_golden,
                     static_from_golden, to_gpu_state)

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

F32_TOL = 1e-5   # relative tolerance of the float32 parity tests
F64_TOL = 1e-12  # float64: the same arithmetic in the same order


def _lib():
    from mbd_icenav_b200 import _abi
    lib = _abi.load_library()
    f = lib.dem_ship_contact_noalloc
    f.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                  C.c_int32, C.c_void_p, C.c_double, C.c_double, C.c_int32, C.c_void_p, C.c_void_p,
                  C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return lib, _abi


def _contact_noalloc(fs, g, prefix, positions, rotations, eta, n=None):
    """Call the new entry point on torch device tensors; returns (rc, pen, normals)."""
    lib, abi = _lib()
    dt = positions.dtype
    dev = positions.device
    st = static_from_golden(g, prefix)
    sd = shipdyn_from_golden(g, prefix)
    polys = torch.as_tensor(np.asarray(st.local_polys_padded, np.float64)).to(dev, dt).contiguous()
    mask = torch.as_tensor(np.asarray(st.poly_mask, bool)).to(dev).contiguous()
    hull = torch.as_tensor(np.asarray(sd.ship_hull_local, np.float64)).to(dev, dt).contiguous()
    n_el = positions.shape[0]
    pen = torch.full((n_el,), float("nan"), dtype=dt, device=dev)
    nrm = torch.full((n_el, 2), float("nan"), dtype=dt, device=dev)
    P = fs.params
    code = abi.DEM_F32 if dt == torch.float32 else abi.DEM_F64
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    rc = lib.dem_ship_contact_noalloc(code, n_el if n is None else n, polys.shape[1], polys.data_ptr(),
                                      mask.data_ptr(), positions.contiguous().data_ptr(),
                                      rotations.contiguous().data_ptr(), hull.shape[0], hull.data_ptr(),
                                      P.half_len, P.half_beam, P.n_edge_samples, eta.contiguous().data_ptr(),
                                      pen.data_ptr(), nrm.data_ptr(), stream)
    torch.cuda.synchronize()
    return rc, pen, nrm


def _state_at(g, prefix, f, dtype):
    """Input state of frame f: the golden output of frame f-1 for the contact inputs."""
    o_st, o_sh = initial_state(g, prefix, dtype)
    if f > 0:
        o_st = o_st._replace(positions=np.asarray(g[f"{prefix}_pos"][f - 1], dtype),
                             rotations=np.asarray(g[f"{prefix}_rot"][f - 1], dtype))
        o_sh = o_sh._replace(eta=np.asarray(g[f"{prefix}_eta"][f - 1], dtype))
    return o_st, o_sh


def _frame_step_pen(fs, g, prefix, f, st, sh, dtype):
    sp, spn, vw, vws = frame_inputs(g, prefix, f)
    d = torch.device("cuda", 0)
    t = lambda a: torch.as_tensor(np.asarray(a, np.float64)).to(d, dtype)
    _, _, diag = fs(st, sh, t(sp), t(spn), t(vw), st.dpdem_floe_eligible, t(vws))
    torch.cuda.synchronize()
    return diag["pen_max"]


def test_noalloc_contact_matches_frame_step_on_two_calls_in_a_row(golden32, golden64):
    cases = [("window", golden32, 0, np.float32, torch.float32, F32_TOL),
             ("small", golden64, 79, np.float64, torch.float64, F64_TOL)]
    for call, (prefix, g, f, npdt, tdt, tol) in enumerate(cases):
        fs = gpu_frame_step(g, prefix, tdt)
        o_st, o_sh = _state_at(g, prefix, f, npdt)
        st, sh = to_gpu_state(o_st, o_sh, tdt)
        want = _frame_step_pen(fs, g, prefix, f, st, sh, tdt).cpu().numpy()
        rc, pen, nrm = _contact_noalloc(fs, g, prefix, st.positions, st.rotations, sh.eta)
        assert rc == 0, (call, rc)
        got = pen.cpu().numpy()
        assert (want > 0).sum() > 0, "the case must contain contacts"
        np.testing.assert_array_equal(got > 0, want > 0, err_msg=f"call {call} ({prefix})")
        assert rel_err(got, want, 1e-6) <= tol, (call, prefix, rel_err(got, want, 1e-6))
        # normals (frame_step does not report them): unit length at every contact,
        # and in float64 the oracle's max-penetration normals
        gn = nrm.cpu().numpy()
        assert np.all(np.isfinite(gn))
        hit = want > 0
        np.testing.assert_allclose(np.hypot(gn[hit, 0], gn[hit, 1]), 1.0, atol=1e-4)
        if npdt == np.float64:
            o = make_oracle(g, prefix, npdt, pair_mode="grid")
            _, o_nx, o_ny = o.ship_contact(o_st.positions, o_st.rotations, *o_sh.eta)
            assert float(np.max(np.abs(gn - np.stack([o_nx, o_ny], -1)))) <= 1e-9
        fs.close()


def test_noalloc_contact_rejects_sizes_beyond_its_scratch(golden64):
    from mbd_icenav_b200 import _abi
    g = golden64
    fs = gpu_frame_step(g, "small", torch.float64)
    o_st, o_sh = _state_at(g, "small", 0, np.float64)
    st, sh = to_gpu_state(o_st, o_sh, torch.float64)
    lib, abi = _lib()
    rc, pen, _ = _contact_noalloc(fs, g, "small", st.positions, st.rotations, sh.eta,
                                  n=262144 + 1)
    assert rc == _abi.DEM_ERR_CAPACITY
    assert torch.isnan(pen).all()  # nothing was written
    fs.close()
