"""Seeded synthetic ice fields for the three plain-DEM workloads.

The reference builds fields from satellite floes or its synthetic map
(``medea_ice_ship/synthetic_map.py:147-189``), tessellates each floe into
Voronoi cells with mirrored seed points (``tessellation.py:7-101``) and bonds
cells whose centroid distance is below ``1.5 (r_i + r_j)``
(``bonds.py:6-16``).  That code needs shapely, which is absent here, so this
module re-implements the same recipe with NumPy/SciPy only:

* convex floes (points on a circle at jittered angles, i.e. convex by
  construction), placed without overlap by rejection sampling on their
  circumscribed disks, largest first;
* per-floe Voronoi tessellation of jittered seed points, the cells bounded by
  mirrored copies of the seeds and clipped to the floe by Sutherland-Hodgman
  (both polygons are convex, so the clip is exact);
* proximity bonds over all cell pairs, in ``(i, j)``, ``i < j`` lexicographic
  order, as the reference's double loop emits them.

Three presets, sized after the plain-DEM workloads:

``small``   150 x 300 m, 3 seven-vertex floes (radius U[10, 20] m), 8 cells
            each (24 elements), h = 1 m, 7-vertex pointed 60 x 12 m hull
            surging at 2 m/s, 300 frames x 10 substeps of 0.005 s;
``medium``  300 x 750 m at 30 %, 400 floes with 5-12 vertices, log-normal
            areas (median 150 m^2, sigma 0.8), h in {0.5, 1.5} m 50:50,
            ~12k cells, uniform 0.2 m/s current, ship at 2 m/s;
``large``   1.5 x 1.5 km at 70 %, power-law floe areas (exponent -1.8 on
            20-20000 m^2), log-normal h (median 1.2 m, sigma 0.4), ~250k
            cells, ship on a seeded piecewise-linear path at 2.5 m/s.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional, Tuple

import numpy as np

from .state import polygon_centroid
from .vessel import ShipProperties, pointed_hull_outline


# ─── Geometry helpers ────────────────────────────────────────────────────────

def convex_floe(rng: np.random.Generator, n_vertices: int, radius: float,
                jitter: float = 0.3) -> np.ndarray:
    """Vertices on a circle at jittered angles (CCW, convex by construction)."""
    base = 2.0 * np.pi * np.arange(n_vertices) / n_vertices
    step = 2.0 * np.pi / n_vertices
    ang = base + rng.uniform(-jitter, jitter, n_vertices) * step
    ang = np.sort(np.mod(ang, 2.0 * np.pi))
    return np.column_stack([radius * np.cos(ang), radius * np.sin(ang)])


def clip_convex(subject, clip) -> Optional[np.ndarray]:
    """Sutherland-Hodgman clip of a polygon by a convex CCW polygon (float math on lists)."""
    out = [(float(p[0]), float(p[1])) for p in subject]
    cl = [(float(p[0]), float(p[1])) for p in clip]
    m = len(cl)
    for k in range(m):
        ax, ay = cl[k]
        bx, by = cl[(k + 1) % m]
        ex, ey = bx - ax, by - ay
        if not out:
            return None
        side = [ex * (py - ay) - ey * (px - ax) for px, py in out]  # >= 0: inside (left)
        if min(side) >= 0.0:
            continue
        res = []
        npts = len(out)
        for i in range(npts):
            p, q = out[i], out[(i + 1) % npts]
            sp, sq = side[i], side[(i + 1) % npts]
            if sp >= 0.0:
                res.append(p)
            if (sp >= 0.0) != (sq >= 0.0):
                t = sp / (sp - sq)
                res.append((p[0] + t * (q[0] - p[0]), p[1] + t * (q[1] - p[1])))
        out = res
    if len(out) < 3:
        return None
    return np.array(out)


def _dedupe(poly, tol: float = 1e-9) -> np.ndarray:
    pts = [(float(p[0]), float(p[1])) for p in poly]
    keep = [pts[0]]
    for p in pts[1:]:
        if math.hypot(p[0] - keep[-1][0], p[1] - keep[-1][1]) > tol:
            keep.append(p)
    if len(keep) > 1 and math.hypot(keep[0][0] - keep[-1][0], keep[0][1] - keep[-1][1]) <= tol:
        keep.pop()
    return np.array(keep)


def _signed_area2(poly) -> float:
    pts = poly.tolist() if isinstance(poly, np.ndarray) else poly
    acc = 0.0
    px, py = pts[-1]
    for qx, qy in pts:
        acc += px * qy - qx * py
        px, py = qx, qy
    return acc


def _area_fast(poly) -> float:
    return 0.5 * abs(_signed_area2(poly))


def tessellate_floe(rng: np.random.Generator, floe: np.ndarray, n_cells: int) -> List[np.ndarray]:
    """Voronoi cells of jittered seeds inside a convex floe, clipped to it."""
    from scipy.spatial import Voronoi

    lo, hi = floe.min(axis=0), floe.max(axis=0)
    w, h = hi - lo
    area = _area_fast(floe)
    if n_cells <= 1:
        return [floe.copy()]
    aspect = max(0.1, w / max(h, 1e-9))
    ny = max(1, int(round(math.sqrt(n_cells / aspect))))
    nx = max(1, int(math.ceil(n_cells / ny)))
    gx = lo[0] + (np.arange(nx) + 0.5) * (w / nx)
    gy = lo[1] + (np.arange(ny) + 0.5) * (h / ny)
    px, py = np.meshgrid(gx, gy, indexing="ij")
    pts = np.column_stack([px.ravel(), py.ravel()])
    pts += rng.uniform(-0.3, 0.3, pts.shape) * np.array([w / nx, h / ny])
    pts = pts[_inside_convex(pts, floe)]
    spacing = 0.5 * math.sqrt(area / n_cells)
    tries = 0
    while len(pts) < n_cells and tries < 50 * n_cells:
        q = rng.uniform(lo, hi, size=(64, 2))
        q = q[_inside_convex(q, floe)]
        for c in q:
            if len(pts) >= n_cells:
                break
            if len(pts) == 0 or np.min(np.sum((pts - c) ** 2, axis=1)) >= spacing ** 2:
                pts = np.vstack([pts, c[None]]) if len(pts) else c[None].copy()
        tries += 64
    if len(pts) < 3:
        return [floe.copy()]
    margin = 2.0 * max(w, h)
    shifts = [(-1, 0), (1, 0), (0, -1), (0, 1), (-1, -1), (-1, 1), (1, -1), (1, 1)]
    allp = np.vstack([pts] + [pts + margin * np.array(s, dtype=float) for s in shifts])
    vor = Voronoi(allp)
    vin = _inside_convex(vor.vertices, floe)
    cells = []
    for i in range(len(pts)):
        region = vor.regions[vor.point_region[i]]
        if -1 in region or len(region) < 3:
            continue
        poly = vor.vertices[region]
        # 2-D qhull regions are ordered around the cell; make them CCW
        if _signed_area2(poly) < 0:
            poly = poly[::-1]
        if vin[region].all():
            clipped = poly
        else:
            clipped = clip_convex(poly, floe)
            if clipped is None:
                continue
            clipped = _dedupe(clipped)
        if len(clipped) < 3 or _area_fast(clipped) < 1e-6:
            continue
        cells.append(np.ascontiguousarray(clipped))
    return cells if cells else [floe.copy()]


def _inside_convex(pts: np.ndarray, poly: np.ndarray) -> np.ndarray:
    ok = np.ones(len(pts), dtype=bool)
    m = len(poly)
    for k in range(m):
        a, b = poly[k], poly[(k + 1) % m]
        ok &= (b[0] - a[0]) * (pts[:, 1] - a[1]) - (b[1] - a[1]) * (pts[:, 0] - a[0]) > 0.0
    return ok


def proximity_bonds(centroids: np.ndarray, radii: np.ndarray, factor: float = 1.5) -> List[Tuple[int, int]]:
    """All (i, j), i < j, with |c_i - c_j| < factor (r_i + r_j), lexicographic order."""
    from scipy.spatial import cKDTree

    n = len(centroids)
    if n < 2:
        return []
    tree = cKDTree(centroids)
    pairs = tree.query_pairs(r=factor * 2.0 * float(radii.max()), output_type="ndarray")
    if len(pairs) == 0:
        return []
    i, j = np.minimum(pairs[:, 0], pairs[:, 1]), np.maximum(pairs[:, 0], pairs[:, 1])
    d = np.linalg.norm(centroids[i] - centroids[j], axis=1)
    keep = d < (radii[i] + radii[j]) * factor
    i, j = i[keep], j[keep]
    order = np.lexsort((j, i))
    return list(zip(i[order].tolist(), j[order].tolist()))


def place_disks(rng: np.random.Generator, radii: np.ndarray, box: Tuple[float, float, float, float],
                gap: float = 0.5, max_tries: int = 400) -> np.ndarray:
    """Random sequential placement of non-overlapping disks, largest first.

    Disks larger than ``big`` are kept in a list tested with NumPy; the rest
    sit in a uniform grid of cell ``2*big``.  Returns centres
    (len(radii), 2); a disk that finds no room gets NaN.
    """
    x0, x1, y0, y1 = box
    order = np.argsort(-radii)
    big = float(np.quantile(radii, 0.9)) if len(radii) > 20 else float(radii.max())
    cell = 2.0 * big + gap
    grid = {}
    big_c = np.zeros((0, 2))
    big_r = np.zeros(0)
    centres = np.full((len(radii), 2), np.nan)
    for idx in order:
        r = float(radii[idx])
        if x1 - x0 < 2 * r or y1 - y0 < 2 * r:
            continue
        cand = rng.uniform([x0 + r, y0 + r], [x1 - r, y1 - r], size=(max_tries, 2))
        if len(big_r):
            d2 = ((cand[:, None, :] - big_c[None, :, :]) ** 2).sum(-1)
            free = ~(d2 < (r + big_r[None, :] + gap) ** 2).any(axis=1)
        else:
            free = np.ones(len(cand), dtype=bool)
        reach = int(math.ceil((r + big + gap) / cell))
        placed = False
        for ci in np.nonzero(free)[0]:
            c = cand[ci]
            gxi, gyi = int(c[0] // cell), int(c[1] // cell)
            ok = True
            for dx in range(-reach, reach + 1):
                for dy in range(-reach, reach + 1):
                    for other in grid.get((gxi + dx, gyi + dy), ()):
                        oc = centres[other]
                        if (oc[0] - c[0]) ** 2 + (oc[1] - c[1]) ** 2 < (r + radii[other] + gap) ** 2:
                            ok = False
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if ok:
                centres[idx] = c
                placed = True
                break
        if not placed:
            continue
        if r > big:
            big_c = np.vstack([big_c, centres[idx][None]])
            big_r = np.append(big_r, r)
        else:
            c = centres[idx]
            grid.setdefault((int(c[0] // cell), int(c[1] // cell)), []).append(idx)
    return centres


# ─── Field assembly ──────────────────────────────────────────────────────────

@dataclass
class IceField:
    """Everything ``build_static_data`` and the drivers need for one scenario."""

    name: str
    polygons: List[np.ndarray]
    centroids: np.ndarray
    bonds: List[Tuple[int, int]]
    thicknesses: np.ndarray
    parent_ids: np.ndarray
    ship_length: float
    ship_beam: float
    ship_props: ShipProperties
    hull_local: Optional[np.ndarray]
    trajectory: np.ndarray            # (n_frames + 2, 3) setpoints [x, y, psi]
    current: Tuple[float, float]      # uniform water velocity [m/s]
    dt: float                         # frame step [s]
    n_ice_steps: int                  # substeps per frame
    n_frames: int
    domain: Tuple[float, float, float, float]
    extra: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return len(self.polygons)

    @property
    def dt_ice(self) -> float:
        return self.dt / self.n_ice_steps

    def setpoints(self, frame0: int, k: int) -> np.ndarray:
        """(k, 6) rows [sp, sp_next] for frames frame0 .. frame0+k-1 (``jax_simulation.py:1107-1119``)."""
        last = len(self.trajectory) - 1
        rows = []
        for f in range(frame0, frame0 + k):
            a = self.trajectory[min(f, last)]
            b = self.trajectory[min(f + 1, last)]
            rows.append(np.concatenate([a, b]))
        return np.array(rows, dtype=np.float64)


def _straight_path(start, heading, speed, dt, n):
    d = np.array([math.cos(heading), math.sin(heading)])
    return np.array([[start[0] + d[0] * speed * dt * i, start[1] + d[1] * speed * dt * i, heading]
                     for i in range(n)])


def _polyline_path(waypoints: np.ndarray, speed: float, dt: float, n: int) -> np.ndarray:
    seg = np.diff(waypoints, axis=0)
    seg_len = np.linalg.norm(seg, axis=1)
    cum = np.concatenate([[0.0], np.cumsum(seg_len)])
    out = []
    for i in range(n):
        s = min(speed * dt * i, cum[-1])
        k = min(int(np.searchsorted(cum, s, side="right")) - 1, len(seg) - 1)
        t = (s - cum[k]) / max(seg_len[k], 1e-12)
        p = waypoints[k] + t * seg[k]
        out.append([p[0], p[1], math.atan2(seg[k][1], seg[k][0])])
    return np.array(out)


def _cells_from_floes(rng, floes, floe_h, cell_area, min_cells):
    polys, cents, parents, hs = [], [], [], []
    for fi, floe in enumerate(floes):
        a = _area_fast(floe)
        nc = max(min_cells, int(round(a / cell_area)))
        for cell in tessellate_floe(rng, floe, nc):
            polys.append(cell)
            cents.append(polygon_centroid(cell))
            parents.append(fi)
            hs.append(floe_h[fi])
    return polys, np.array(cents), np.array(parents, dtype=np.int32), np.array(hs, dtype=np.float64)


def _finish(name, polys, cents, parents, hs, traj, current, dt, k, n_frames, domain,
            ship_length=60.0, ship_beam=12.0, draft=4.0, hull=None, extra=None) -> IceField:
    areas = np.array([_area_fast(p) for p in polys])
    radii = np.sqrt(areas / np.pi)
    bonds = proximity_bonds(cents, radii, 1.5)
    props = ShipProperties(length=ship_length, beam=ship_beam, draft=draft)
    if hull is None:
        hull = pointed_hull_outline(ship_length, ship_beam)
    return IceField(name=name, polygons=polys, centroids=cents, bonds=bonds, thicknesses=hs,
                    parent_ids=parents, ship_length=ship_length, ship_beam=ship_beam,
                    ship_props=props, hull_local=hull, trajectory=traj, current=current,
                    dt=dt, n_ice_steps=k, n_frames=n_frames, domain=domain, extra=extra or {})


def make_small_field(seed: int = 0, n_frames: int = 300) -> IceField:
    """150 x 300 m, three 7-gon floes of 8 cells each, pointed hull at 2 m/s."""
    rng = np.random.default_rng(seed)
    W, H = 150.0, 300.0
    radii = rng.uniform(10.0, 20.0, 3)
    centres = place_disks(rng, radii, (0.0, W, 60.0, H), gap=2.0)
    floes = [convex_floe(rng, 7, r) + c for r, c in zip(radii, centres)]
    polys, cents, parents, hs = _cells_from_floes(rng, floes, np.ones(3), 1e9, 8)
    # ship starts just south of the lowest floe, bow +y, and surges into it
    k0 = int(np.argmin(centres[:, 1]))
    start = (float(centres[k0, 0]), float(centres[k0, 1] - radii[k0] - 32.0))
    traj = _straight_path(start, math.pi / 2, 2.0, 0.05, n_frames + 2)
    return _finish("small", polys, cents, parents, hs, traj, (0.0, 0.0), 0.05, 10, n_frames,
                   (0.0, W, 0.0, H))


def make_medium_field(seed: int = 0, n_frames: int = 2000, cell_area: float = 6.6) -> IceField:
    """300 x 750 m at 30 %, 400 floes, ~12k cells, 0.2 m/s current."""
    rng = np.random.default_rng(seed)
    W, H = 300.0, 750.0
    areas = np.exp(np.log(150.0) + 0.8 * rng.standard_normal(400))
    nv = rng.integers(5, 13, 400)
    base = [convex_floe(rng, int(k), 1.0) for k in nv]
    scale = np.sqrt(areas / np.array([_area_fast(b) for b in base]))
    centres = place_disks(rng, scale, (0.0, W, 100.0, H), gap=1.0)
    ok = ~np.isnan(centres[:, 0])
    floes = [b * s + c for b, s, c, good in zip(base, scale, centres, ok) if good]
    h = np.where(rng.random(len(floes)) < 0.5, 0.5, 1.5)
    polys, cents, parents, hs = _cells_from_floes(rng, floes, h, cell_area, 2)
    traj = _straight_path((W / 2, 40.0), math.pi / 2, 2.0, 0.05, n_frames + 2)
    return _finish("medium", polys, cents, parents, hs, traj, (0.2, 0.0), 0.05, 10, n_frames,
                   (0.0, W, 0.0, H), extra={"floes": len(floes)})


def make_large_field(seed: int = 0, n_frames: int = 1000, cell_area: float = 6.2,
                     side: float = 1500.0, concentration: float = 0.70) -> IceField:
    """1.5 x 1.5 km at ~70 %, power-law floe areas, ~250k cells."""
    rng = np.random.default_rng(seed)
    a_lo, a_hi, alpha = 20.0, 20000.0, -1.8
    target = concentration * side * side
    # inverse-CDF sampling of p(A) ~ A^alpha on [a_lo, a_hi]
    e = alpha + 1.0
    areas = []
    total = 0.0
    while total < target * 1.02:
        u = rng.random(4096)
        a = (a_lo ** e + u * (a_hi ** e - a_lo ** e)) ** (1.0 / e)
        for v in a:
            areas.append(v)
            total += v
            if total >= target * 1.02:
                break
    areas = np.array(areas)
    nv = rng.integers(5, 13, len(areas))
    base = [convex_floe(rng, int(k), 1.0) for k in nv]
    scale = np.sqrt(areas / np.array([_area_fast(b) for b in base]))
    centres = place_disks(rng, scale, (0.0, side, 0.0, side), gap=0.3, max_tries=60)
    ok = ~np.isnan(centres[:, 0])
    floes = [b * s + c for b, s, c, good in zip(base, scale, centres, ok) if good]
    h = np.exp(np.log(1.2) + 0.4 * rng.standard_normal(len(floes)))
    polys, cents, parents, hs = _cells_from_floes(rng, floes, h, cell_area, 2)
    # seeded piecewise-linear path across the field
    ys = np.linspace(-40.0, side + 40.0, 6)
    xs = side / 2 + rng.uniform(-0.25, 0.25, 6) * side
    xs[0] = side / 2
    way = np.column_stack([xs, ys])
    traj = _polyline_path(way, 2.5, 0.05, n_frames + 2)
    covered = float(sum(_area_fast(f) for f in floes)) / (side * side)
    return _finish("large", polys, cents, parents, hs, traj, (0.0, 0.0), 0.05, 10, n_frames,
                   (0.0, side, 0.0, side), extra={"floes": len(floes), "concentration": covered})


def morton_order(points: np.ndarray, cell: float) -> np.ndarray:
    """Permutation sorting points along a Z-order (Morton) curve of square cells."""
    q = np.floor((points - points.min(axis=0)) / cell).astype(np.int64)
    q = np.clip(q, 0, (1 << 20) - 1)

    def spread(v):
        v = (v | (v << 16)) & 0x0000FFFF0000FFFF
        v = (v | (v << 8)) & 0x00FF00FF00FF00FF
        v = (v | (v << 4)) & 0x0F0F0F0F0F0F0F0F
        v = (v | (v << 2)) & 0x3333333333333333
        v = (v | (v << 1)) & 0x5555555555555555
        return v

    code = spread(q[:, 0]) | (spread(q[:, 1]) << 1)
    return np.argsort(code, kind="stable")


def spatially_sorted(field: IceField, cell: float = 4.0) -> IceField:
    """The same field with its elements renumbered in Morton order of their centroids.

    Element order does not change the physics (bond and pair lists are
    renumbered with it); it decides memory locality of the per-element gathers.
    """
    perm = morton_order(field.centroids, cell)
    inv = np.empty_like(perm)
    inv[perm] = np.arange(len(perm))
    bonds = [(int(min(inv[i], inv[j])), int(max(inv[i], inv[j]))) for i, j in field.bonds]
    bonds.sort()
    import dataclasses
    return dataclasses.replace(field, polygons=[field.polygons[k] for k in perm],
                               centroids=field.centroids[perm], bonds=bonds,
                               thicknesses=field.thicknesses[perm], parent_ids=field.parent_ids[perm])


def make_field(name: str, seed: int = 0, **kw) -> IceField:
    return {"small": make_small_field, "medium": make_medium_field,
            "large": make_large_field}[name](seed=seed, **kw)


def hexagon_fixture(n_frames: int = 30, dt: float = 0.05) -> IceField:
    """Three r = 3 m hexagons at x = -10, 0, 10 bonded in a chain; 15 x 5 m ship moving +x.

    The canonical small fixture of the reference's own tests
    (``test_jax_full_scan.py:187-230``).
    """
    ang = np.linspace(0, 2 * np.pi, 7)[:-1]
    hexp = np.column_stack([3.0 * np.cos(ang), 3.0 * np.sin(ang)])
    cents = np.array([[-10.0, 0.0], [0.0, 0.0], [10.0, 0.0]])
    polys = [hexp + c for c in cents]
    traj = np.array([[-25.0 + i * 0.5, 0.0, 0.0] for i in range(n_frames + 2)])
    props = ShipProperties(length=15.0, beam=5.0, draft=2.5)
    return IceField(name="hexagons", polygons=polys, centroids=cents, bonds=[(0, 1), (1, 2)],
                    thicknesses=np.ones(3), parent_ids=np.arange(3, dtype=np.int32),
                    ship_length=15.0, ship_beam=5.0, ship_props=props, hull_local=None,
                    trajectory=traj, current=(0.0, 0.0), dt=dt, n_ice_steps=1,
                    n_frames=n_frames, domain=(-20.0, 20.0, -10.0, 10.0))
