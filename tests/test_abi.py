"""The C-ABI library loads and exports every entry point its header declares (no GPU needed)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT


def _declared(header="dem_b200.h", prefix="dem_"):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(rf"^\s*(?:int|const char\*)\s+({prefix}\w+)\s*\(", src, flags=re.M)))


def test_header_declares_the_boundary():
    names = _declared()
    for need in ("dem_create", "dem_frame_step", "dem_scan_segment", "dem_destroy", "dem_get_error",
                 "dem_sync_status"):
        assert need in names


def test_library_exports_every_declared_symbol():
    from mbd_icenav_b200 import _abi, build
    build.build_library()
    lib = ctypes.CDLL(build.LIB_PATH)
    for name in _declared():
        assert hasattr(lib, name), name
    assert set(_abi.EXPORTS) <= set(_declared())
    assert lib.dem_version is not None


def test_library_exports_every_surrogate_symbol():
    """The surrogate's kernels (include/surrogate_b200.h) live in the same library."""
    from mbd_icenav_b200 import _abi, build
    build.build_library()
    lib = ctypes.CDLL(build.LIB_PATH)
    names = _declared("surrogate_b200.h", "sg_")
    assert "sg_gemm" in names
    for name in names:
        assert hasattr(lib, name), name
    assert set(_abi.SG_EXPORTS) == set(names)


def test_struct_layout_matches_header():
    """ctypes mirrors must have the header's field order (checked by name against the source)."""
    from mbd_icenav_b200 import _abi
    src = open(os.path.join(ROOT, "include", "dem_b200.h")).read()
    body = src[src.index("typedef struct DemParams"):src.index("} DemParams;")]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    fields = []
    for line in body.splitlines()[1:]:
        line = line.strip().rstrip(";")
        if not line:
            continue
        decl = line.split(None, 1)[1]
        for part in decl.split(","):
            fields.append(part.strip().split("[")[0])
    assert fields == [f for f, _ in _abi.DemParams._fields_]


def test_null_arguments_are_rejected_without_a_gpu():
    from mbd_icenav_b200 import _abi
    lib = _abi.load_library()
    assert lib.dem_create(None, None, 0, 0, None) == _abi.DEM_ERR_INVALID
    assert lib.dem_frame_step(None, None, None, None, None, None, None, None, None, None, None, None) \
        == _abi.DEM_ERR_INVALID
    assert lib.dem_destroy(None) == _abi.DEM_OK


def test_sweep_features_rejects_bad_arguments_without_a_gpu():
    """dem_rollout_sweep_features checks its sizes and pointers before any CUDA call."""
    from mbd_icenav_b200 import _abi
    lib = _abi.load_library()
    f32 = _abi.DEM_F32
    p = 16  # any non-null value: nothing is dereferenced before the checks fail
    args = dict(dtype=f32, Q=4, H=8, eta0=p, hist=p, n=10, pos=p, radii=p, mass=p, nb=0, bi=None, bj=None,
                hl=30.0, hw=6.0, dt=0.05, out=p)

    def call(**kw):
        a = dict(args, **kw)
        return lib.dem_rollout_sweep_features(a["dtype"], a["Q"], a["H"], a["eta0"], a["hist"], a["n"], a["pos"],
                                              a["radii"], a["mass"], a["nb"], a["bi"], a["bj"], a["hl"], a["hw"],
                                              a["dt"], a["out"], None)

    bad = [dict(dtype=7), dict(Q=0), dict(H=0), dict(H=513), dict(n=65537), dict(n=-1), dict(dt=0.0),
           dict(hl=-1.0), dict(eta0=None), dict(out=None), dict(pos=None), dict(nb=3), dict(hist=None)]
    for kw in bad:
        assert call(**kw) == _abi.DEM_ERR_INVALID, kw
