"""Particle geometry for workloads the reference reads from particle files.

The aggregate workload is 8 hexagonal columns (diameter 20 um, length 60 um)
with seed-drawn orientations, assembled so that each new column touches the
cluster without overlapping it (coordinates on a power-of-two lattice, see
`column_aggregate`), written in the reference's particle-file format (`--particle-file`, README.md "particle file": CONCAVE flag,
AGGREGATE flag and facets per component, beta/gamma symmetry in degrees,
then facets as blank-line separated vertex lists wound so that every facet
normal points outward).
"""
from __future__ import annotations

import numpy as np


def hex_prism(diameter: float, length: float) -> list[np.ndarray]:
    """Facets of a hexagonal column centred at the origin with its axis on z:
    vertex-to-vertex diameter `diameter` (the reference's Hexagonal
    convention), bases first and last, outward winding."""
    r, h = diameter / 2.0, length / 2.0
    ang = np.arange(6) * np.pi / 3.0
    ring = np.stack([r * np.cos(ang), r * np.sin(ang)], axis=1)
    top = np.column_stack([ring, np.full(6, h)])                 # counter-clockwise seen from +z
    bottom = np.column_stack([ring[::-1], np.full(6, -h)])       # clockwise seen from +z
    facets = [top]
    for i in range(6):
        j = (i + 1) % 6
        facets.append(np.array([[ring[i, 0], ring[i, 1], -h], [ring[j, 0], ring[j, 1], -h],
                                [ring[j, 0], ring[j, 1], h], [ring[i, 0], ring[i, 1], h]]))
    facets.append(bottom)
    return facets


def triangulated(facets: list[np.ndarray]) -> list[np.ndarray]:
    """Each convex facet as a fan of triangles with the same winding.  The
    reference's particle-file loader snaps coordinates to a power-of-two grid
    of 2^-40 of the particle extent and then requires every facet planar to
    2^-40 of the facet size, which a generically rotated polygon of more than
    three vertices cannot meet; coplanar triangles cover the same aperture."""
    out = []
    for f in facets:
        for i in range(1, len(f) - 1):
            out.append(np.array([f[0], f[i], f[i + 1]]))
    return out


def facet_normal(f: np.ndarray) -> np.ndarray:
    n = np.cross(f[1] - f[0], f[2] - f[1])
    return n / np.linalg.norm(n)


def random_rotation(rng) -> np.ndarray:
    """Uniformly distributed rotation matrix (unit quaternion from normals)."""
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


class Convex:
    """A convex polyhedron: facets, vertices, face normals, edge directions."""

    def __init__(self, facets: list[np.ndarray]):
        self.facets = facets
        self.verts = np.unique(np.round(np.concatenate(facets), 12), axis=0)
        self.normals = np.array([facet_normal(f) for f in facets])
        edges = []
        for f in facets:
            for i in range(len(f)):
                e = f[(i + 1) % len(f)] - f[i]
                edges.append(e / np.linalg.norm(e))
        self.edges = np.array(edges)

    def moved(self, R: np.ndarray, t: np.ndarray) -> "Convex":
        return Convex([f @ R.T + t for f in self.facets])


def separated(a: Convex, b: Convex, tol: float = 0.0) -> bool:
    """Separating-axis test: True when some axis (a face normal of either or
    a cross product of their edge directions) separates the two by more than
    tol."""
    axes = [a.normals, b.normals]
    cr = np.cross(a.edges[:, None, :], b.edges[None, :, :]).reshape(-1, 3)
    nrm = np.linalg.norm(cr, axis=1)
    axes.append(cr[nrm > 1e-9] / nrm[nrm > 1e-9, None])
    ax = np.concatenate(axes)
    pa, pb = a.verts @ ax.T, b.verts @ ax.T
    gap = np.maximum(pb.min(axis=0) - pa.max(axis=0), pa.min(axis=0) - pb.max(axis=0))
    return bool(np.any(gap > tol))


def min_separation(a: Convex, b: Convex) -> float:
    """Largest separating-axis gap (> 0: apart by at least that much along
    some axis; <= 0: the polyhedra overlap or touch)."""
    axes = [a.normals, b.normals]
    cr = np.cross(a.edges[:, None, :], b.edges[None, :, :]).reshape(-1, 3)
    nrm = np.linalg.norm(cr, axis=1)
    axes.append(cr[nrm > 1e-9] / nrm[nrm > 1e-9, None])
    ax = np.concatenate(axes)
    pa, pb = a.verts @ ax.T, b.verts @ ax.T
    return float(np.max(np.maximum(pb.min(axis=0) - pa.max(axis=0), pa.min(axis=0) - pb.max(axis=0))))


def _rational_rotation(rng, K: int = 64):
    """A seed-drawn rotation with rational entries, R = M / n, M integer and
    n = a^2 + b^2 + c^2 + d^2 for the integer quaternion (a, b, c, d) nearest
    K times a uniformly drawn unit quaternion."""
    while True:
        q = rng.normal(size=4)
        q = np.rint(K * q / np.linalg.norm(q)).astype(np.int64)
        n = int(np.dot(q, q))
        if n > 0:
            break
    a, b, c, d = (int(v) for v in q)
    M = np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                  [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                  [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]],
                 dtype=np.int64)
    return M, n


def _lattice_prism(diameter: float, length: float, unit: float) -> list[np.ndarray]:
    """hex_prism with every coordinate rounded to an integer number of
    `unit` (integer arrays); the hexagon stays regular to unit/diameter."""
    r, h = diameter / 2.0, length / 2.0
    R, Rh, Ry, H = (int(round(x / unit)) for x in (r, r / 2.0, r * np.sqrt(3.0) / 2.0, h))
    ring = np.array([[R, 0], [Rh, Ry], [-Rh, Ry], [-R, 0], [-Rh, -Ry], [Rh, -Ry]], dtype=np.int64)
    top = np.column_stack([ring, np.full(6, H)])
    bottom = np.column_stack([ring[::-1], np.full(6, -H)])
    facets = [top]
    for i in range(6):
        j = (i + 1) % 6
        facets.append(np.array([[ring[i, 0], ring[i, 1], -H], [ring[j, 0], ring[j, 1], -H],
                                [ring[j, 0], ring[j, 1], H], [ring[i, 0], ring[i, 1], H]],
                               dtype=np.int64))
    facets.append(bottom)
    return facets


def column_aggregate(n: int = 8, diameter: float = 20.0, length: float = 60.0, seed: int = 2024,
                     gap: float = 0.02) -> list[Convex]:
    """n hexagonal columns with seed-drawn orientations; each new column comes
    in from a seed-drawn direction towards the cluster centroid and stops at
    first contact (bisection to 1e-6 um), then backs off until every column
    is at least `gap` away, so it touches the cluster to within `gap` without
    overlapping any column.

    Coordinates are exact multiples of a power-of-two unit (2 q, q the
    reference loader's snapping quantum for this extent, 2^(ilogb(extent) -
    40)): rotations are rational, R = M / n, applied in integer arithmetic to
    prisms whose coordinates are integer multiples of n 2 q.  The loader's
    centring and snapping then leave every coordinate unchanged, and every
    facet (8 per column) stays exactly planar."""
    extent = 2.0 * np.hypot(diameter, length) * np.sqrt(n)        # first guess
    for _attempt in range(3):
        q = 2.0 ** (int(np.floor(np.log2(extent))) - 40)
        unit = 2.0 * q
        rng = np.random.default_rng(seed)
        comps: list[Convex] = []
        placed = []
        reach = 2.0 * np.hypot(diameter, length) * n
        for i in range(n):
            M, nn = _rational_rotation(rng)
            body = _lattice_prism(diameter, length, nn * unit)        # integers, units nn*unit
            rot = [(f @ M.T) for f in body]                            # integers, units unit
            rot_f = [f.astype(np.float64) * unit for f in rot]
            if i == 0:
                shift = np.zeros(3, dtype=np.int64)
            else:
                d = rng.normal(size=3)
                d /= np.linalg.norm(d)
                c0 = np.mean([c.verts.mean(axis=0) for c in comps], axis=0)
                lo, hi = 0.0, reach
                while hi - lo > 1e-6:
                    mid = 0.5 * (lo + hi)
                    cand = Convex([f + c0 + d * mid for f in rot_f])
                    if all(separated(cand, c) for c in comps):
                        hi = mid
                    else:
                        lo = mid
                t = hi
                while True:
                    shift = np.rint((c0 + d * t) / unit).astype(np.int64)
                    cand = Convex([f + shift * unit for f in rot_f])
                    if min(min_separation(cand, c) for c in comps) >= gap:
                        break
                    t += 0.25 * gap
            placed.append([f + shift for f in rot])
            comps.append(Convex([f.astype(np.float64) * unit for f in placed[-1]]))
        allv = np.concatenate([np.concatenate(p) for p in placed])
        span = (allv.max(axis=0) - allv.min(axis=0)) * unit
        got = float(np.sqrt(np.sum(span * span)))
        if int(np.floor(np.log2(got))) == int(np.floor(np.log2(extent))):
            # centre on an even multiple of the unit so the loader's midpoint
            # is a lattice point
            mid2 = allv.max(axis=0) + allv.min(axis=0)              # 2 * midpoint, units
            centre = mid2 // 2
            return [Convex([(f - centre).astype(np.float64) * unit for f in p]) for p in placed]
        extent = got
    raise RuntimeError("aggregate extent does not settle on one power-of-two scale")


def write_particle_file(path: str, comps: list[Convex], concave: int = 1,
                        beta_sym_deg: float = 180.0, gamma_sym_deg: float = 360.0) -> None:
    """Reference particle-file text (aggregate of convex components)."""
    per = len(comps[0].facets)
    with open(path, "w") as f:
        f.write("# aggregate of %d convex components, %d facets each\n" % (len(comps), per))
        f.write("%d\n1 %d\n%.6g %.6g\n" % (concave, per, beta_sym_deg, gamma_sym_deg))
        for c in comps:
            for fac in c.facets:
                f.write("\n")
                for v in fac:
                    f.write("%.17g %.17g %.17g\n" % tuple(v))
