"""Conformal periodic tetrahedral meshes of a slab stack with one polygonal hole.

The batched workload uses random polygonal holes (3-8 vertices, side wall
80-90 deg) cut through the absorber of the slab stack.  The reference lofts
such a frustum as an exact polytope: the cross-section at height z is the
base polygon under a uniform mitre offset of |z - z0| / tan(alpha), every
vertex moving along its angle bisector so that each side wall is one planar
quad (src/lithofem/meshgen.py:139-166, src/lithofem/geometry.py:1-12,
175-194), and meshes it with gmsh.  gmsh is not available here; this module
builds the same geometry as a structured, conformal mesh:

* a 2D mesh of the periodic cell.  Rays from the hole centre c pass through
  every polygon vertex and through boundary points chosen in periodic pairs
  (x = 0 <-> x = Lx, y = 0 <-> y = Ly).  Between the polygon and the box the
  strips between consecutive rays are cut into quads (straight polygon and
  box pieces, since all polygon vertices and box corners sit on rays).
  Inside the polygon, nested rings (the polygon scaled about c, with point
  counts shrinking towards c) are joined by a zipper triangulation, ending
  in a fan at c;
* extrusion through z levels that contain every interface; each layer of
  triangular prisms is cut into 3 tetrahedra by the minimum-vertex-id rule
  on the periodic (identified) vertex ids, which makes neighbouring prisms
  agree on every quad-face diagonal, across the periodic boundary too;
* node motion with z: polygon-boundary nodes keep their edge parameter on
  the mitre-offset polygon, ring nodes follow the moved boundary, box nodes
  stay, so the hole walls are the reference's planar quads.  Every tet's
  orientation is checked against the unmoved extrusion (no tangling).

Element attributes follow the region table of ``Stack.regions`` (slab-major,
background first, then the hole, PML slabs last).
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .mesh import Stack, TetMesh, _axis_nodes


@dataclass(frozen=True)
class PolyHole:
    """Polygonal frustum: CCW base polygon ``verts`` at z0, height h > 0,
    side-wall angle alpha (deg; < 90 narrows the section away from the
    base), star-shaped about its centre (cx, cy)."""

    cx: float
    cy: float
    verts: tuple
    z0: float
    h: float
    alpha: float
    eps: complex

    @property
    def z_lo(self) -> float:
        return min(self.z0, self.z0 + self.h)

    @property
    def z_hi(self) -> float:
        return max(self.z0, self.z0 + self.h)

    def inset(self, z) -> np.ndarray:
        """Inward mitre offset distance of the section at height z."""
        z = np.asarray(z, dtype=float)
        t = 1.0 / math.tan(math.radians(self.alpha)) if self.alpha != 90 else 0.0
        return np.clip(np.abs(z - self.z0), 0.0, abs(self.h)) * t

    def mitre(self) -> np.ndarray:
        """(nv, 2) vertex velocities of a unit inward mitre offset."""
        V = np.asarray(self.verts, dtype=float)
        E = np.roll(V, -1, axis=0) - V
        N = np.stack([-E[:, 1], E[:, 0]], axis=1) / np.linalg.norm(E, axis=1)[:, None]  # inward (CCW)
        Np = np.roll(N, 1, axis=0)  # normal of the edge ending at vertex i
        return (Np + N) / (1.0 + np.sum(Np * N, axis=1))[:, None]

    def section(self, d: float) -> np.ndarray:
        return np.asarray(self.verts, dtype=float) + d * self.mitre()

    def area(self, d: float = 0.0) -> float:
        P = self.section(d)
        x, y = P[:, 0], P[:, 1]
        return 0.5 * float(np.sum(x * np.roll(y, -1) - np.roll(x, -1) * y))


def random_hole(rng: np.random.Generator, lx: float, ly: float, z0: float, h: float,
                nv: int, alpha: float, eps: complex = 1.0 + 0j,
                r_range: tuple[float, float] = (0.18, 0.34)) -> PolyHole:
    """A star-shaped polygon with nv vertices around a jittered cell centre;
    radii U(r_range) x min(lx, ly), angular gaps bounded away from 0 and pi."""
    L = min(lx, ly)
    while True:
        gaps = rng.uniform(0.5, 1.5, nv)
        gaps = gaps / gaps.sum() * 2 * math.pi
        if gaps.max() >= 0.8 * math.pi:
            continue
        th = rng.uniform(0, 2 * math.pi) + np.concatenate([[0.0], np.cumsum(gaps)[:-1]])
        r = rng.uniform(*r_range, nv) * L
        cx = 0.5 * lx + rng.uniform(-0.04, 0.04) * L
        cy = 0.5 * ly + rng.uniform(-0.04, 0.04) * L
        V = np.stack([cx + r * np.cos(th), cy + r * np.sin(th)], axis=1)
        hole = PolyHole(cx, cy, tuple(map(tuple, V)), z0, h, alpha, eps)
        if _section_ok(hole, float(hole.inset(z0 + h)), lx, ly):
            return hole


def _section_ok(hole: PolyHole, dmax: float, lx: float, ly: float) -> bool:
    """The offset sections stay star-shaped about c, CCW, inside the cell."""
    c = np.array([hole.cx, hole.cy])
    for d in np.linspace(0.0, dmax, 9):
        P = hole.section(d)
        if P[:, 0].min() < 0.08 * lx or P[:, 0].max() > 0.92 * lx:
            return False
        if P[:, 1].min() < 0.08 * ly or P[:, 1].max() > 0.92 * ly:
            return False
        Q = np.roll(P, -1, axis=0)
        # c strictly left of every edge (star-shaped about c, with margin)
        cr = (Q[:, 0] - P[:, 0]) * (c[1] - P[:, 1]) - (Q[:, 1] - P[:, 1]) * (c[0] - P[:, 0])
        if (cr <= 0.05 * np.linalg.norm(Q - P, axis=1) * min(lx, ly)).any():
            return False
    return True


def _ray_box(c, ang, lx, ly):
    """Distance from c along angle ang to the box boundary."""
    dx, dy = math.cos(ang), math.sin(ang)
    ts = []
    if dx > 1e-15:
        ts.append((lx - c[0]) / dx)
    if dx < -1e-15:
        ts.append(-c[0] / dx)
    if dy > 1e-15:
        ts.append((ly - c[1]) / dy)
    if dy < -1e-15:
        ts.append(-c[1] / dy)
    return min(ts)


def _ray_poly(c, ang, V):
    """(edge index, edge parameter) where the ray from c hits polygon V."""
    d = np.array([math.cos(ang), math.sin(ang)])
    n = len(V)
    best = None
    for i in range(n):
        a, b = V[i], V[(i + 1) % n]
        e = b - a
        den = d[0] * (-e[1]) - d[1] * (-e[0])
        if abs(den) < 1e-14:
            continue
        rhs = a - c
        t = (rhs[0] * (-e[1]) - rhs[1] * (-e[0])) / den   # along the ray
        u = (d[0] * rhs[1] - d[1] * rhs[0]) / den          # along the edge
        if t > 0 and -1e-12 <= u <= 1 + 1e-12:
            if best is None or t < best[0]:
                best = (t, i, min(max(u, 0.0), 1.0))
    if best is None:
        raise RuntimeError("ray misses the polygon")
    return best[1], best[2]


def _fill(req: list[float], h: float) -> list[float]:
    req = sorted(set(round(v, 12) for v in req))
    out = [req[0]]
    for a, b in zip(req[:-1], req[1:]):
        n = max(1, int(math.ceil((b - a) / h - 1e-9)))
        out.extend(a + (b - a) * np.arange(1, n + 1) / n)
    return out


def build_poly_mesh(stack: Stack, hole: PolyHole, h: float) -> TetMesh:
    """Mesh ``stack`` (domain plus both PML slabs) around ``hole`` with
    target edge length h."""
    lx, ly = stack.lx, stack.ly
    c = np.array([hole.cx, hole.cy])
    V = np.asarray(hole.verts, dtype=float)
    nv = len(V)

    # ---- boundary points in periodic pairs, including the vertex-ray hits
    xr, yr = [0.0, lx], [0.0, ly]
    for k in range(nv):
        ang = math.atan2(V[k, 1] - c[1], V[k, 0] - c[0])
        t = _ray_box(c, ang, lx, ly)
        p = c + t * np.array([math.cos(ang), math.sin(ang)])
        if abs(p[0]) < 1e-9 or abs(p[0] - lx) < 1e-9:
            yr.append(float(p[1]))
        else:
            xr.append(float(p[0]))
    Y = _fill(yr, h)
    X = _fill(xr, h)
    bpts = []  # (x, y, canonical key)
    for y in Y:
        bpts.append((0.0, y))
        bpts.append((lx, y))
    for x in X[1:-1]:
        bpts.append((x, 0.0))
        bpts.append((x, ly))
    bpts = np.array(bpts)
    ang_b = np.arctan2(bpts[:, 1] - c[1], bpts[:, 0] - c[0])
    order = np.argsort(ang_b, kind="stable")
    bpts, ang_b = bpts[order], ang_b[order]
    nr = len(bpts)

    # ---- 2D nodes.  ring-0 (polygon) nodes are parameterised by (edge, u)
    # so that they can follow the mitre-offset polygon in z.
    hit = [_ray_poly(c, a, V) for a in ang_b]
    pe = np.array([e for e, _ in hit])
    pu = np.array([u for _, u in hit])
    # snap vertex rays exactly onto the vertices
    for k in range(nv):
        a = math.atan2(V[k, 1] - c[1], V[k, 0] - c[0])
        j = int(np.argmin(np.abs(np.angle(np.exp(1j * (ang_b - a))))))
        pe[j], pu[j] = k, 0.0
    rpoly = np.array([np.linalg.norm(V[e] + u * (V[(e + 1) % nv] - V[e]) - c)
                      for e, u in zip(pe, pu)])
    rbox = np.linalg.norm(bpts - c, axis=1)
    n_out = max(1, int(round(float(np.mean(rbox - rpoly)) / h)))
    K = max(1, int(round(float(np.mean(rpoly)) / h)))

    # node records: kind 0 = ring node (ring k, edge e, u) incl. polygon
    # (k = 0) and centre (k = K); kind 1 = exterior (ray i, level j, 1..n_out)
    nodes = []
    ring_ids = []
    # ring 0
    ring_ids.append(list(range(nr)))
    for i in range(nr):
        nodes.append((0, 0, int(pe[i]), float(pu[i])))
    # arc-length parameterisation of the polygon for inner rings
    elen = np.linalg.norm(np.roll(V, -1, axis=0) - V, axis=1)
    perim = float(elen.sum())
    cum = np.concatenate([[0.0], np.cumsum(elen)])
    s0 = cum[pe] + pu * elen[pe]  # arc position of ring-0 nodes
    for k in range(1, K):
        frac = 1.0 - k / K
        # point spacing ~h along every ring: the centre fan stays small
        nk = max(3, min(nr, int(round(perim * frac / h))))
        start = s0[0]
        ids = []
        for m in range(nk):
            s = (start + perim * m / nk) % perim
            e = int(np.searchsorted(cum, s, side="right") - 1)
            e = min(e, nv - 1)
            u = (s - cum[e]) / elen[e]
            ids.append(len(nodes))
            nodes.append((0, k, e, float(u)))
        ring_ids.append(ids)
    centre = len(nodes)
    nodes.append((0, K, 0, 0.0))
    ext = np.zeros((nr, n_out + 1), dtype=np.int64)
    ext[:, 0] = np.arange(nr)
    for i in range(nr):
        for j in range(1, n_out + 1):
            ext[i, j] = len(nodes)
            nodes.append((1, i, j, 0.0))
    nn = len(nodes)

    def pos2d(d: float) -> np.ndarray:
        """2D node positions for a mitre offset d of the polygon."""
        P = hole.section(d)
        out = np.zeros((nn, 2))
        for idx, (kind, a, b, u) in enumerate(nodes):
            if kind == 0:
                if a == K:
                    out[idx] = c
                    continue
                q = P[b] + u * (P[(b + 1) % nv] - P[b])
                out[idx] = c + (1.0 - a / K) * (q - c)
        for i in range(nr):
            q = out[ext[i, 0]]
            for j in range(1, n_out + 1):
                w = j / n_out
                out[ext[i, j]] = (1.0 - w) * q + w * bpts[i]
        return out

    P0 = pos2d(0.0)

    # ---- triangles (CCW), zone 0 = inside the polygon, 1 = outside
    tris, zone = [], []
    for i in range(nr):
        i2 = (i + 1) % nr
        for j in range(n_out):
            a0, a1, b0, b1 = ext[i, j], ext[i, j + 1], ext[i2, j], ext[i2, j + 1]
            tris += [(a0, a1, b1), (a0, b1, b0)]
            zone += [1, 1]
    angs = [np.arctan2(P0[ids, 1] - c[1], P0[ids, 0] - c[0]) for ids in ring_ids]
    two_pi = 2 * math.pi
    for k in range(K - 1):
        A, B = ring_ids[k], ring_ids[k + 1]
        ta, tb = angs[k], angs[k + 1]
        na, nb = len(A), len(B)
        # unwrapped angles, A from its first node, B from its node nearest it
        al = ta[0] + np.mod(ta - ta[0], two_pi)
        al = np.append(al, ta[0] + two_pi)
        j0 = int(np.argmin(np.abs(np.angle(np.exp(1j * (tb - ta[0]))))))
        tb = np.roll(tb, -j0)
        Bs = [B[(j0 + m) % nb] for m in range(nb)]
        be0 = ta[0] + float(np.angle(np.exp(1j * (tb[0] - ta[0]))))
        be = be0 + np.mod(tb - tb[0], two_pi)
        be = np.append(be, be0 + two_pi)
        ia = ib = 0
        while ia < na or ib < nb:
            if ib == nb or (ia < na and al[ia + 1] <= be[ib + 1]):
                tris.append((A[ia], A[(ia + 1) % na], Bs[ib % nb]))
                ia += 1
            else:
                tris.append((A[ia % na], Bs[(ib + 1) % nb], Bs[ib]))
                ib += 1
            zone.append(0)
    last = ring_ids[K - 1]
    for m in range(len(last)):
        tris.append((last[m], last[(m + 1) % len(last)], centre))
        zone.append(0)
    tris = np.array(tris, dtype=np.int64)
    zone = np.array(zone)
    ar = _tri_area(P0, tris)
    if (ar <= 0).any():
        raise RuntimeError("inverted triangle in the base mesh")

    # ---- periodic identification of box nodes
    topo = np.arange(nn)
    key = {}
    for i in range(nr):
        nid = ext[i, n_out]
        x, y = bpts[i]
        cx_ = 0.0 if abs(x - lx) < 1e-9 else x
        cy_ = 0.0 if abs(y - ly) < 1e-9 else y
        kk = (round(cx_, 9), round(cy_, 9))
        if kk in key:
            topo[nid] = key[kk]
        else:
            key[kk] = nid
    # compact topological ids
    uniq, topo = np.unique(topo, return_inverse=True)
    nv2 = len(uniq)

    # ---- z levels through every interface
    t = stack.pml_thick
    zb = [stack.z_min - t, stack.z_min, stack.z_max, stack.z_max + t] + stack.slabs
    zb += [hole.z_lo, hole.z_hi]
    zn = _axis_nodes(zb, h)
    nz = len(zn) - 1

    pos = np.stack([pos2d(float(hole.inset(z))) for z in zn])       # (nz+1, nn, 2)
    pos_ref = np.broadcast_to(P0, pos.shape)

    # prisms -> 3 tets (minimum-vertex-id rule on periodic ids)
    tid = topo[tris]                                   # (nt, 3)
    o = np.argsort(tid, axis=1, kind="stable")
    u = np.take_along_axis(tris, o, axis=1)            # 2D node ids sorted by topo id
    pat = np.array([[(0, 0), (1, 0), (2, 0), (2, 1)],
                    [(0, 0), (1, 0), (1, 1), (2, 1)],
                    [(0, 0), (0, 1), (1, 1), (2, 1)]])  # (corner, level offset)
    ne = len(tris) * 3 * nz
    tv = np.zeros((ne, 4), dtype=np.int64)
    xv = np.zeros((ne, 4, 3))
    xr = np.zeros((ne, 4, 3))
    ezone = np.zeros(ne, dtype=np.int64)
    m = 0
    for k in range(nz):
        for q in range(3):
            cols = u[:, pat[q, :, 0]]                  # (nt, 4) 2D node ids
            lev = k + pat[q, :, 1]                     # (4,)
            sl = slice(m, m + len(tris))
            tv[sl] = lev[None, :] * nv2 + topo[cols]
            xv[sl, :, :2] = pos[lev[None, :], cols]
            xv[sl, :, 2] = zn[lev][None, :]
            xr[sl, :, :2] = pos_ref[lev[None, :], cols]
            xr[sl, :, 2] = zn[lev][None, :]
            ezone[sl] = zone
            m += len(tris)
    vol = _tet_vol(xv)
    vref = _tet_vol(xr)
    if (np.sign(vol) != np.sign(vref)).any() or (np.abs(vol) < 1e-12 * h ** 3).any():
        raise RuntimeError("tangled or degenerate element after wall motion")

    # ---- attributes
    regs = stack.regions()
    cen = xv.mean(axis=1)
    zc = cen[:, 2]
    s = stack.slabs
    slab = np.clip(np.searchsorted(np.array(s[1:-1]), zc, side="right"), 0, len(s) - 2)
    attr = np.zeros(ne, dtype=np.int32)
    for ridx, r in enumerate(regs, start=1):
        if r["kind"] == "background":
            attr[(slab == r["slab"]) & (zc >= stack.z_min) & (zc <= stack.z_max)] = ridx
    for ridx, r in enumerate(regs, start=1):
        if r["kind"] != "frustum":
            continue
        inside = ((slab == r["slab"]) & (zc >= stack.z_min) & (zc <= stack.z_max)
                  & (zc >= hole.z_lo) & (zc <= hole.z_hi) & (ezone == 0))
        attr[inside] = ridx
    attr[zc < stack.z_min] = len(regs) - 1
    attr[zc > stack.z_max] = len(regs)
    if (attr == 0).any():  # pragma: no cover - geometry bug guard
        raise RuntimeError("unassigned elements")
    return TetMesh(tv=tv, xv=xv, attr=attr, nv=int(nv2 * (nz + 1)), grid=(nr, K, nz))


def _tri_area(P: np.ndarray, tris: np.ndarray) -> np.ndarray:
    a, b, c = P[tris[:, 0]], P[tris[:, 1]], P[tris[:, 2]]
    return 0.5 * ((b[:, 0] - a[:, 0]) * (c[:, 1] - a[:, 1]) - (b[:, 1] - a[:, 1]) * (c[:, 0] - a[:, 0]))


def _tet_vol(x: np.ndarray) -> np.ndarray:
    a = x[:, 1] - x[:, 0]
    b = x[:, 2] - x[:, 0]
    c = x[:, 3] - x[:, 0]
    return np.einsum("ij,ij->i", a, np.cross(b, c)) / 6.0
