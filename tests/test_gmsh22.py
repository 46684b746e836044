"""The Gmsh 2.2 + $Periodic mesh input (lithofem_b200.gmsh22), the reference
solver's ``mesh.per.msh`` format (src/lithofem/meshgen.py:112-122,
485-506).

* Written and read back, a mesh gives the same topological vertices,
  element coordinates and attributes, and so the same space and per-mesh
  data (every AsmData array equal).
* A file in the layout the reference's writer produces -- node ids that are
  not contiguous, boundary triangles, an ``Affine`` line, corner nodes
  identified through a chain (y-image -> x-image -> master) -- reads to the
  same vertex partition.
* Malformed input is refused with a message.
"""

from __future__ import annotations

import re

import numpy as np
import pytest

from lithofem_b200 import configs, gmsh22, space
from lithofem_b200.mesh_poly import build_poly_mesh
from lithofem_b200.mesh import build_mesh


def _ad_equal(a, b):
    for f in ("dof", "sign", "fopack", "J", "Jinv", "detJ", "v0", "attr", "ess"):
        x, y = getattr(a, f, None), getattr(b, f, None)
        if x is None and y is None:
            continue
        assert np.array_equal(np.asarray(x), np.asarray(y)), f
    assert a.height == b.height and a.ne == b.ne


@pytest.mark.parametrize("kind,p", [("grating", 2), ("hole", 3), ("slab", 1)])
def test_round_trip_gives_the_same_space(tmp_path, kind, p):
    c = configs.small_case(kind, p, 6.0, seed=None)
    f = tmp_path / "m.per.msh"
    gmsh22.write_msh22(c.mesh, f)
    m = gmsh22.read_msh22(f)
    assert np.array_equal(m.tv, c.mesh.tv) and np.array_equal(m.xv, c.mesh.xv)
    assert np.array_equal(m.attr, c.mesh.attr) and m.nv == c.mesh.nv
    _ad_equal(space.build_asm_data(m, p, c.prob), space.build_asm_data(c.mesh, p, c.prob))


def test_round_trip_of_a_polygon_hole_mesh(tmp_path):
    rng = np.random.default_rng(4)
    st = configs.poly_hole_stack(rng, lx=24.0, ly=24.0, z_max=30.0, t_range=(10.0, 14.0),
                                 pml_wl=0.3)
    mesh = build_poly_mesh(st, st.frustums[0], 4.0)
    f = tmp_path / "poly.per.msh"
    gmsh22.write_msh22(mesh, f)
    m = gmsh22.read_msh22(f)
    assert np.array_equal(m.tv, mesh.tv) and np.array_equal(m.xv, mesh.xv)
    assert np.array_equal(m.attr, mesh.attr)


def _reference_layout(text: str, lx: float, ly: float) -> str:
    """Rewrite a written file into the reference writer's layout: node ids
    x 3 + 5, boundary triangles added, an Affine line, and the corner
    images (x = lx, y = ly) paired with their y-image (x = lx, y = 0), which
    is itself the x-image of the master."""
    lines = text.splitlines()
    i = lines.index("$Nodes")
    nn = int(lines[i + 1])
    pos = {}
    for ln in lines[i + 2:i + 2 + nn]:
        t, x, y, z = ln.split()
        pos[int(t)] = (float(x), float(y), float(z))
    new = lambda t: 3 * int(t) + 5  # noqa: E731
    out = []
    section = None
    per = []
    for ln in lines:
        if ln.startswith("$"):
            section = ln[1:]
            out.append(ln)
            continue
        f = ln.split()
        if section == "Nodes" and len(f) == 4:
            out.append(" ".join([str(new(f[0]))] + f[1:]))
        elif section == "Elements" and len(f) > 4:
            out.append(" ".join(f[:5] + [str(new(v)) for v in f[5:]]))
        elif section == "Periodic" and len(f) == 2:
            per.append((int(f[0]), int(f[1])))
        else:
            out.append(ln)
    # boundary triangles: the first face of the first two tetrahedra
    ei = out.index("$Elements")
    ne = int(out[ei + 1])
    tets = out[ei + 2:ei + 2 + ne]
    tris = []
    for k, ln in enumerate(tets[:2]):
        f = ln.split()
        tris.append(f"{ne + k + 1} 2 2 1 7 {f[5]} {f[6]} {f[7]}")
    out[ei + 1] = str(ne + len(tris))
    out[ei + 2 + ne:ei + 2 + ne] = tris
    # chained corners
    by_pos = {tuple(np.round(pos[s], 9)): s for s, _ in per}
    pairs = []
    for s, m in per:
        x, y, z = pos[s]
        if abs(x - lx) < 1e-9 and abs(y - ly) < 1e-9:
            mid = by_pos.get(tuple(np.round((lx, 0.0, z), 9)))
            if mid is not None:
                m = mid
        pairs.append((new(s), new(m)))
    pi = out.index("$Periodic")
    out[pi + 1:out.index("$EndPeriodic")] = (
        ["1", "2 2 1", "Affine 1 0 0 -1 0 1 0 0 0 0 1 0 0 0 0 1", str(len(pairs))]
        + [f"{s} {m}" for s, m in pairs])
    return "\n".join(out) + "\n"


def test_reference_layout_with_chained_corners(tmp_path):
    c = configs.small_case("hole", 2, 6.0, seed=None)
    f = tmp_path / "a.per.msh"
    gmsh22.write_msh22(c.mesh, f)
    g = tmp_path / "b.per.msh"
    text = _reference_layout(f.read_text(), c.stack.lx, c.stack.ly)
    assert "Affine" in text and re.search(r"^\d+ 2 2 1 7 ", text, re.M)
    body = text[text.index("$Periodic"):].splitlines()[5:]
    pairs = [tuple(map(int, ln.split())) for ln in body if len(ln.split()) == 2]
    slaves = {s for s, _ in pairs}
    assert sum(m in slaves for _, m in pairs) > 0     # some masters are slaves: chains
    g.write_text(text)
    m = gmsh22.read_msh22(g)
    assert m.ne == c.mesh.ne and m.nv == c.mesh.nv
    assert np.array_equal(m.xv, c.mesh.xv) and np.array_equal(m.attr, c.mesh.attr)
    # the same partition of the element vertices into topological vertices
    a, b = c.mesh.tv.reshape(-1), m.tv.reshape(-1)
    fwd = np.full(c.mesh.nv, -1)
    fwd[a] = b
    assert np.array_equal(fwd[a], b) and len(np.unique(fwd)) == c.mesh.nv


def test_malformed_input_is_refused(tmp_path):
    mesh = build_mesh(configs.small_case("slab", 1, 0.0).stack, 3.0)
    f = tmp_path / "m.msh"
    gmsh22.write_msh22(mesh, f)
    text = f.read_text()
    cases = {
        "4.1 0 8": "is not 2.x",
        "2.2 1 8": "binary",
    }
    for fmt, msg in cases.items():
        g = tmp_path / "bad.msh"
        g.write_text(text.replace("2.2 0 8", fmt, 1))
        with pytest.raises(ValueError, match=msg):
            gmsh22.read_msh22(g)
    g.write_text(text.replace("$EndNodes\n", "", 1))
    with pytest.raises(ValueError, match="no \\$EndNodes"):
        gmsh22.read_msh22(g)
    g.write_text(text.replace("$MeshFormat", "$Format", 1).replace("$EndMeshFormat", "$EndFormat"))
    with pytest.raises(ValueError, match="no \\$MeshFormat"):
        gmsh22.read_msh22(g)
