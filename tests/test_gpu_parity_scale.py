"""GPU parity at the bench's scale, fp32, against the fp32 oracle.

The bench times the f32 frame kernel on the whole 245k-element large field
(64-entry hash buckets, CTA-wide list rebuilds, lazy escapes on a 1.5 km
domain).  Here that same handle (the bench's own constructor, capacities and
skin) first advances the field with the ship inside it, then one frame at a
time is checked against the oracle from the identical fp32 state:

* every IceState / ShipState field per entry within 1e-5 of its own change
  over the frame (floor: fp32 rounding of the value, and twice the fp32
  oracle's own error against the float64 oracle from the same input), masks
  bit-equal;
* the ice-ice contact set of every substep bit-equal to the oracle's
  all-pairs set (restated broad phase: exact, see the oracle's header);
* the ship contact mask, force magnitudes and ship force.

The medium field (12k elements, 0.2 m/s current) gets the same check.  The
oracle's frame on the large field takes ~12 s on one core (fp32 and fp64 each).
"""
import os
import sys

import numpy as np
import pytest

from helpers import assert_frame_matches, contact_sets_match

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _oracle(field, dtype):
    from mbd_icenav_b200.config import SimulationConfig
    from mbd_icenav_b200.state import build_static_arrays, ship_dynamics_arrays
    from mbd_icenav_b200.vessel import SupplyVessel
    from oracle.dem_oracle import Oracle, params_from_config
    import bench
    cfg = SimulationConfig()
    sa = build_static_arrays(field.polygons, field.centroids, field.bonds, field.thicknesses, field.parent_ids,
                             cfg, dilation=0.05)
    sd = ship_dynamics_arrays(field.ship_props, cfg, field.ship_length, field.ship_beam, field.hull_local)
    sv = SupplyVessel(mass=field.ship_props.mass, length=field.ship_length)
    p = params_from_config(cfg, field.ship_length, field.ship_beam, bench.N_SUB, bench.DT, bench.DT / bench.N_SUB,
                           False, sv.T_n)
    return Oracle(sa, sd, p, sv.B, dtype, pair_mode="grid")


def _check_field(name, advance, frames):
    sys.path.insert(0, ROOT)
    import bench
    from helpers import to_np_state
    from oracle.dem_oracle import OShip, OState
    field = bench.load_field(name, 0)
    dev = torch.device("cuda", 0)
    fs, st, sh, _ = bench.build_stepper(field, "f32", dev, 64, 0.8)
    n = fs.n
    vw_row = torch.tensor(field.current, dtype=torch.float32, device=dev).expand(n, 2)
    sp = torch.as_tensor(field.setpoints(bench.START_FRAME, advance + frames), dtype=torch.float32, device=dev)
    # advance with the ship in the field (the bench's own frames, one launch)
    st, sh, _ = fs.scan_segment(st, sh, sp[:advance], vw_row.expand(advance, n, 2).contiguous(), history=False)
    o = _oracle(field, np.float32)
    o64 = _oracle(field, np.float64)  # the fp32 reference's own error, per entry
    rec = fs.record_contacts(capacity=1 << 22)
    vw_np = vw_row.cpu().numpy()
    sp_np = sp.cpu().numpy()
    n_active, n_contacts = [], 0
    for f in range(advance, advance + frames):
        ice_in, ship_in = to_np_state(st, sh)
        o_in = OState(*ice_in)
        o_sh_in = OShip(*ship_in)
        o.contact_log = []
        o_st, o_sh, o_diag = o.frame_step(o_in, o_sh_in, sp_np[f, :3], sp_np[f, 3:], vw_np, o_in.dpdem_floe_eligible)
        d64 = lambda t: type(t)(*[np.asarray(a, np.float64) if np.asarray(a).dtype != bool else a for a in t])
        o64_st, o64_sh, _ = o64.frame_step(d64(o_in), d64(o_sh_in), sp_np[f, :3], sp_np[f, 3:], vw_np,
                                           o_in.dpdem_floe_eligible)
        st, sh, diag = fs(st, sh, sp[f, :3], sp[f, 3:], vw_row.contiguous(), st.dpdem_floe_eligible)
        ice, ship = to_np_state(st, sh)
        worst = assert_frame_matches(ice, ship, o_st, o_sh, o_in, o_sh_in, diag, o_diag, where=f"{name} frame {f}",
                                     o_ice64=o64_st, o_ship64=o64_sh)
        sets, raw = rec.substeps(fs.n_ice_steps)
        n_contacts += contact_sets_match(sets, raw, o.contact_log, o_st.elem_active, where=f"{name} frame {f}")
        n_active.append(int(o_st.elem_active.sum()))
        print(name, "frame", f, "active", n_active[-1], "worst error / tolerance:",
              {k: f"{v:.2e}" for k, v in worst.items()})
    fs.stop_recording()
    assert min(n_active) > 0 and n_contacts > 0, "the ship must be in the ice"
    print(name, "contact pairs with an active end compared:", n_contacts)
    fs.close()


def test_large_field_f32_frames_match_oracle():
    """The bench's workload: 245k elements, ship 100 frames into its timed stretch."""
    _check_field("large", advance=100, frames=2)


def test_medium_field_with_current_f32_frames_match_oracle():
    """12k elements under the uniform 0.2 m/s current, ship pushing into the floes."""
    _check_field("medium", advance=150, frames=3)
