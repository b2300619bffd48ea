"""State and static-data containers with the reference's array layout.

Field names, order, shapes and meaning follow ``medea_ice_ship/jax_ice_state.py``:

* ``IceState``         (``jax_ice_state.py:31-44``)  mutable ice state;
* ``ShipState``        (``jax_ice_state.py:47-52``)  ship pose/velocity/RPM/integral;
* ``IceStaticData``    (``jax_ice_state.py:59-96``)  immutable geometry/material/topology;
* ``ShipDynamicsData`` (``jax_ice_state.py:99-116``) vessel matrices and hull outline.

Arrays are torch tensors (CUDA for the product path); ``(n, 2)`` fields are
row-major interleaved xy, booleans are ``torch.bool`` (one byte), indices are
int32.  Any DLPack producer (a JAX array included) can be turned into these
fields zero-copy with ``torch.from_dlpack``.

The builders restate ``build_static_data`` (``jax_ice_state.py:150-243``),
``build_initial_ice_state`` (``:246-267``), ``build_ship_dynamics_data``
(``:270-343``) and ``build_initial_ship_state`` (``:346-355``) in NumPy
float64, then move the result to the device in the requested dtype.

One deliberate difference: the reference materialises all ``n(n-1)/2``
ice-ice pairs in ``pair_i``/``pair_j`` (``:212-214``), which is 250 GB at
250k elements.  Here the pair list is implicit ("all pairs"): ``pair_i`` and
``pair_j`` are ``None`` and the GPU broad phase finds exactly the pairs of
that list whose disks overlap, which are the only pairs that contribute.
"""
from __future__ import annotations

from typing import List, NamedTuple, Optional, Sequence, Tuple

import numpy as np

from .config import DEFAULT_MATERIAL, IceMaterial, cfg_get
from .vessel import SupplyVessel, tapered_hull_outline


class IceState(NamedTuple):
    positions: object            # (n, 2)
    velocities: object           # (n, 2)
    rotations: object            # (n,)
    angular_vels: object         # (n,)
    submergence: object          # (n,)
    bond_intact: object          # (n_bonds,) bool
    bond_damage: object          # (n_bonds,)
    bond_delta_m_0: object       # (n_bonds,)
    bond_delta_m_max: object     # (n_bonds,)
    bond_delta_s: object         # (n_bonds,)
    elem_active: object          # (n,) bool
    dpdem_floe_eligible: object  # (n_floes,) bool


class ShipState(NamedTuple):
    eta: object       # (3,) [x, y, psi]
    nu: object        # (3,) [u, v, r]
    n_actual: object  # (6,)
    e_int: object     # (3,)


class IceStaticData(NamedTuple):
    local_polys_padded: object  # (n, max_V, 2)
    poly_mask: object           # (n, max_V) bool
    poly_n_verts: object        # (n,) int32
    masses: object
    inertia: object
    radii: object
    areas: object
    thicknesses: object
    bond_i: object              # (n_bonds,) int32
    bond_j: object
    rest_lengths: object
    bond_strengths: object
    bond_areas: object
    sigma_bar_bond: object
    pair_i: object              # None: implicit all-pairs list
    pair_j: object
    initial_floe_of: object     # (n,) int32
    k_n: float
    k_s: float


class ShipDynamicsData(NamedTuple):
    M3inv: object
    D3: object
    mass: float
    Izz: float
    Kp: object
    Kd: object
    Ki: object
    B_pinv: object
    n_max: object
    ship_hull_local: object  # (S, 2)


# ─── NumPy (float64) builders ────────────────────────────────────────────────

def polygon_area(verts) -> float:
    """Shoelace area, |sum x_i y_{i+1} - x_{i+1} y_i| / 2, accumulated in vertex
    order in float64 like ``geometry.py:6-14``."""
    v = np.asarray(verts, dtype=np.float64)
    xs = v[:, 0].tolist()
    ys = v[:, 1].tolist()
    m = len(xs)
    acc = 0.0
    for k in range(m):
        k1 = (k + 1) % m
        acc += xs[k] * ys[k1]
        acc -= xs[k1] * ys[k]
    return abs(acc) / 2


def polygon_centroid(verts: np.ndarray) -> np.ndarray:
    """Vertex mean, which the reference uses as the local-frame origin (``geometry.py:17-18``)."""
    return np.mean(np.asarray(verts, dtype=np.float64), axis=0)


def pad_polygons(local_polys: Sequence[np.ndarray]):
    """Pad to (n, max_V, 2) by repeating each polygon's last real vertex (``jax_ice_state.py:123-147``)."""
    n = len(local_polys)
    n_verts = np.array([len(p) for p in local_polys], dtype=np.int32)
    max_v = int(n_verts.max()) if n else 0
    padded = np.zeros((n, max_v, 2), dtype=np.float64)
    mask = np.zeros((n, max_v), dtype=bool)
    for e, poly in enumerate(local_polys):
        k = len(poly)
        padded[e, :k] = poly
        padded[e, k:] = poly[-1]
        mask[e, :k] = True
    return padded, mask, n_verts


def build_static_arrays(polygons: List[np.ndarray], centroids: np.ndarray,
                        bonds: Sequence[Tuple[int, int]], thicknesses: np.ndarray,
                        parent_ids: Optional[np.ndarray], cfg,
                        material: IceMaterial = DEFAULT_MATERIAL,
                        dilation: float = 0.0) -> IceStaticData:
    """Static data as float64 NumPy arrays (``jax_ice_state.py:150-243``).

    ``dilation`` is added to the contact radii after every other quantity is
    derived, i.e. it is ``static._replace(radii=radii + dilation)``: masses,
    inertia and bond strengths use the undilated equivalent-disk radius.
    """
    n = len(polygons)
    centroids = np.asarray(centroids, dtype=np.float64).reshape(n, 2)
    thicknesses = np.asarray(thicknesses, dtype=np.float64).reshape(n)
    areas = np.array([polygon_area(p) for p in polygons], dtype=np.float64)
    radii = np.sqrt(areas / np.pi)
    masses = areas * thicknesses * material.ice_density
    inertia = np.maximum(0.5 * masses * radii ** 2, 1e-10)
    local = [(np.asarray(p, dtype=np.float64) - polygon_centroid(p)) for p in polygons]
    padded, mask, n_verts = pad_polygons(local)

    bonds = list(bonds)
    nb = len(bonds)
    if nb:
        bi = np.array([b[0] for b in bonds], dtype=np.int32)
        bj = np.array([b[1] for b in bonds], dtype=np.int32)
        rest = np.linalg.norm(centroids[bi] - centroids[bj], axis=1)
        h = np.minimum(thicknesses[bi], thicknesses[bj])
        w = np.minimum((radii[bi] + radii[bj]) / 2, cfg_get(cfg, "max_bond_width"))
        strengths = material.breaking_force(h, w)
        b_areas = w * h
        sigma_bar = np.maximum(strengths / np.maximum(b_areas, 1e-10), 1e6)
    else:
        bi = np.zeros(0, np.int32); bj = np.zeros(0, np.int32)
        rest = strengths = b_areas = sigma_bar = np.zeros(0, np.float64)

    nu_r = cfg_get(cfg, "poisson_ratio")
    E = material.youngs_modulus
    pref = E * (1.0 - nu_r) / ((1.0 + nu_r) * (1.0 - 2.0 * nu_r))
    k_n = pref
    k_s = pref * (1.0 - 2.0 * nu_r) / (2.0 * (1.0 - nu_r))

    floe_of = (np.asarray(parent_ids, dtype=np.int32) if parent_ids is not None
               else np.arange(n, dtype=np.int32))
    return IceStaticData(
        local_polys_padded=padded, poly_mask=mask, poly_n_verts=n_verts,
        masses=masses, inertia=inertia, radii=radii + dilation, areas=areas,
        thicknesses=thicknesses, bond_i=bi, bond_j=bj, rest_lengths=rest,
        bond_strengths=strengths, bond_areas=b_areas, sigma_bar_bond=sigma_bar,
        pair_i=None, pair_j=None, initial_floe_of=floe_of,
        k_n=float(k_n), k_s=float(k_s))


def initial_ice_state_arrays(n: int, centroids: np.ndarray, n_bonds: int,
                             initial_floe_of: np.ndarray) -> IceState:
    """Zero-velocity, undamaged, all-frozen state (``jax_ice_state.py:246-267``)."""
    n_floes = int(np.max(initial_floe_of)) + 1 if n > 0 else 0
    f = np.float64
    return IceState(
        positions=np.asarray(centroids, dtype=f).reshape(n, 2).copy(),
        velocities=np.zeros((n, 2), f), rotations=np.zeros(n, f),
        angular_vels=np.zeros(n, f), submergence=np.zeros(n, f),
        bond_intact=np.ones(n_bonds, bool), bond_damage=np.zeros(n_bonds, f),
        bond_delta_m_0=np.zeros(n_bonds, f), bond_delta_m_max=np.zeros(n_bonds, f),
        bond_delta_s=np.zeros(n_bonds, f), elem_active=np.zeros(n, bool),
        dpdem_floe_eligible=np.zeros(n_floes, bool))


def ship_dynamics_arrays(ship_props, cfg, ship_length: float, ship_beam: float,
                         hull_local: Optional[np.ndarray] = None) -> ShipDynamicsData:
    """Vessel matrices, pole-placement gains and hull outline (``jax_ice_state.py:270-343``).

    ``hull_local`` overrides the default 62-point tapered outline (used by the
    7-vertex pointed hull of the seeded benchmark fields).
    """
    m = ship_props.mass
    izz = (1.0 / 12.0) * m * (ship_length ** 2 + ship_beam ** 2)
    v = SupplyVessel(mass=m, length=ship_length)
    m3d = np.diag(np.diag(v.M3))
    d3d = np.diag(np.diag(v.D3))
    kp = v.wn @ v.wn @ m3d
    kd = 2.0 * v.zeta @ v.wn @ m3d - d3d
    ki = np.zeros((3, 3))
    b_pinv = v.B.T @ np.linalg.inv(v.B @ v.B.T)
    hull = tapered_hull_outline(ship_length, ship_beam) if hull_local is None else np.asarray(hull_local, np.float64)
    return ShipDynamicsData(M3inv=v.M3inv, D3=v.D3, mass=float(v.mass), Izz=float(izz),
                            Kp=kp, Kd=kd, Ki=ki, B_pinv=b_pinv, n_max=v.n_max.copy(),
                            ship_hull_local=hull)


def initial_ship_state_arrays(ship_pos, ship_heading: float) -> ShipState:
    """Zero-velocity ship at ``ship_pos`` (``jax_ice_state.py:346-355``)."""
    return ShipState(eta=np.array([ship_pos[0], ship_pos[1], ship_heading], dtype=np.float64),
                     nu=np.zeros(3), n_actual=np.zeros(6), e_int=np.zeros(3))


# ─── Device transfer ─────────────────────────────────────────────────────────

def _to_torch(x, dtype, device):
    import torch
    if x is None or isinstance(x, float):
        return x
    a = np.asarray(x)
    if a.dtype == bool:
        return torch.from_numpy(np.ascontiguousarray(a)).to(device=device)
    if a.dtype.kind in "iu":
        return torch.from_numpy(np.ascontiguousarray(a.astype(np.int32))).to(device=device)
    return torch.from_numpy(np.ascontiguousarray(a)).to(device=device, dtype=dtype)


def to_device(tup, dtype=None, device="cuda"):
    """Move every array field of a NamedTuple to torch on ``device``; floats become ``dtype``."""
    import torch
    dtype = dtype or torch.float32
    return type(tup)(*[_to_torch(v, dtype, device) for v in tup])


def to_numpy(tup):
    """Copy every tensor field of a NamedTuple back to NumPy."""
    out = []
    for v in tup:
        if hasattr(v, "detach"):
            out.append(v.detach().cpu().numpy())
        else:
            out.append(v)
    return type(tup)(*out)


def build_static_data(polygons, centroids, bonds, thicknesses, parent_ids, cfg,
                      material: IceMaterial = DEFAULT_MATERIAL, dilation: float = 0.0,
                      dtype=None, device="cuda") -> IceStaticData:
    """Drop-in for ``build_static_data`` returning device tensors."""
    return to_device(build_static_arrays(polygons, centroids, bonds, thicknesses,
                                         parent_ids, cfg, material, dilation), dtype, device)


def build_initial_ice_state(n, centroids, n_bonds, initial_floe_of, dtype=None, device="cuda") -> IceState:
    return to_device(initial_ice_state_arrays(n, centroids, n_bonds, np.asarray(initial_floe_of)),
                     dtype, device)


def build_ship_dynamics_data(ship_props, cfg, ship_length, ship_beam, hull_local=None,
                             dtype=None, device="cuda") -> ShipDynamicsData:
    return to_device(ship_dynamics_arrays(ship_props, cfg, ship_length, ship_beam, hull_local),
                     dtype, device)


def build_initial_ship_state(ship_pos, ship_heading, dtype=None, device="cuda") -> ShipState:
    return to_device(initial_ship_state_arrays(ship_pos, ship_heading), dtype, device)
