"""Gmsh 2.2 ASCII meshes with a ``$Periodic`` section.

This is the reference solver's mesh input: ``mesh.per.msh``, the 2.2
sibling of the 4.1 contract file with the side-surface groups dropped and a
``$Periodic`` section appended (src/lithofem/meshgen.py:112-122 writes the
blocks ``dim slave master`` / ``n`` / ``n`` node pairs, :485-506 the files;
solver/lithofem_solve.cpp:469 loads it through MFEM, which identifies every
slave node with its master).

``read_msh22`` turns such a file into a :class:`TetMesh`: tetrahedra
(element type 4) with their first tag, the physical group, as the region
attribute; every ``$Periodic`` pair identifies a slave node with its master,
chains (a corner node that is the slave of a node that is itself a slave)
followed to their last master; the masters, in ascending file order, are
the topological vertices.  Other element types (the boundary triangles)
are skipped: the space finds its boundary faces as the faces that one
element alone references, which is where the reference's PEC groups lie.

``write_msh22`` is the inverse for a TetMesh: one node per distinct
(topological vertex, position) pair, the first position of each vertex (in
element order) numbered 1..nv as its master and the periodic images after
it, and one ``$Periodic`` block that pairs every image with its master.
Reading a written mesh gives back the same ``tv``, ``xv`` and ``attr``.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np

from .mesh import TetMesh

TET = 4


def _sections(text: str) -> dict[str, list[str]]:
    """Lines of every $Name ... $EndName section (the first of each name)."""
    out: dict[str, list[str]] = {}
    lines = text.splitlines()
    i = 0
    while i < len(lines):
        ln = lines[i].strip()
        if ln.startswith("$") and not ln.startswith("$End"):
            name = ln[1:]
            j = i + 1
            while j < len(lines) and lines[j].strip() != "$End" + name:
                j += 1
            if j == len(lines):
                raise ValueError(f"section ${name} has no $End{name}")
            out.setdefault(name, lines[i + 1:j])
            i = j + 1
        else:
            i += 1
    return out


def _find(parent: np.ndarray, a: int) -> int:
    r = a
    while parent[r] != r:
        r = parent[r]
    while parent[a] != r:
        parent[a], a = r, parent[a]
    return r


def read_msh22(path: str | Path) -> TetMesh:
    """A Gmsh 2.2 ASCII mesh (with or without $Periodic) as a TetMesh."""
    sec = _sections(Path(path).read_text())
    if "MeshFormat" not in sec:
        raise ValueError("not a Gmsh mesh: no $MeshFormat")
    fmt = sec["MeshFormat"][0].split()
    if len(fmt) < 2 or not fmt[0].startswith("2."):
        raise ValueError(f"Gmsh format {fmt[0] if fmt else '?'} is not 2.x (write the 2.2 sibling)")
    if fmt[1] != "0":
        raise ValueError("binary Gmsh 2.2 files are not supported (write ASCII)")
    if "Nodes" not in sec or "Elements" not in sec:
        raise ValueError("mesh without $Nodes or $Elements")
    nl = sec["Nodes"]
    nn = int(nl[0])
    if len(nl) < nn + 1:
        raise ValueError(f"$Nodes announces {nn} nodes, holds {len(nl) - 1}")
    raw = np.array(" ".join(nl[1:nn + 1]).split(), dtype=np.float64).reshape(nn, 4)
    ids = raw[:, 0].astype(np.int64)
    xyz = raw[:, 1:]
    index = {int(t): i for i, t in enumerate(ids)}
    if len(index) != nn:
        raise ValueError("repeated node id in $Nodes")

    el = sec["Elements"]
    ne_all = int(el[0])
    tets, attrs = [], []
    for ln in el[1:ne_all + 1]:
        f = ln.split()
        if int(f[1]) != TET:
            continue
        ntag = int(f[2])
        nodes = f[3 + ntag:3 + ntag + 4]
        if len(nodes) != 4:
            raise ValueError(f"tetrahedron {f[0]} has {len(nodes)} nodes")
        try:
            tets.append([index[int(v)] for v in nodes])
        except KeyError as e:
            raise ValueError(f"tetrahedron {f[0]} references unknown node {e.args[0]}") from None
        attrs.append(int(f[3]) if ntag > 0 else 1)
    if not tets:
        raise ValueError("mesh without tetrahedra")
    tn = np.array(tets, dtype=np.int64)

    # periodic identification: slave -> master, chains followed
    parent = np.arange(nn, dtype=np.int64)
    if "Periodic" in sec:
        pl = sec["Periodic"]
        nb = int(pl[0])
        k = 1
        for _ in range(nb):
            if len(pl[k].split()) != 3:
                raise ValueError(f"bad $Periodic block header {pl[k]!r}")
            k += 1
            if pl[k].split()[0] == "Affine":
                k += 1
            npair = int(pl[k])
            k += 1
            for ln in pl[k:k + npair]:
                s_id, m_id = ln.split()[:2]
                try:
                    s, m = index[int(s_id)], index[int(m_id)]
                except KeyError as e:
                    raise ValueError(f"$Periodic pair names unknown node {e.args[0]}") from None
                rs, rm = _find(parent, s), _find(parent, m)
                if rs != rm:
                    parent[rs] = rm
            k += npair
    roots = np.array([_find(parent, i) for i in range(nn)], dtype=np.int64)
    used = np.unique(roots[tn.reshape(-1)])
    topo = np.full(nn, -1, dtype=np.int64)
    topo[used] = np.arange(len(used))
    tv = topo[roots[tn]]
    return TetMesh(tv=tv, xv=xyz[tn], attr=np.array(attrs, dtype=np.int64), nv=len(used))


def write_msh22(mesh: TetMesh, path: str | Path) -> None:
    """Write a TetMesh as Gmsh 2.2 ASCII with a $Periodic section."""
    ne = mesh.ne
    tv = np.asarray(mesh.tv, dtype=np.int64).reshape(-1)
    xv = np.asarray(mesh.xv, dtype=np.float64).reshape(-1, 3)
    # distinct (vertex, position) occurrences in element order
    key = np.concatenate([tv[:, None].astype(np.float64), xv], axis=1)
    _, first, inv = np.unique(key, axis=0, return_index=True, return_inverse=True)
    inv = inv.reshape(-1)
    occ_order = np.argsort(first, kind="stable")       # occurrences by first appearance
    occ_vertex = tv[first]
    occ_pos = xv[first]
    # master of each vertex: its first occurrence; node ids 1..nv for masters
    # (by vertex), nv+1.. for the images (by first appearance)
    nv = int(mesh.nv)
    master_occ = np.full(nv, -1, dtype=np.int64)
    for o in occ_order:
        v = occ_vertex[o]
        if master_occ[v] < 0:
            master_occ[v] = o
    if (master_occ < 0).any():
        raise ValueError("topological vertex without an element")
    node_id = np.zeros(len(first), dtype=np.int64)
    node_id[master_occ] = np.arange(1, nv + 1)
    is_img = np.ones(len(first), dtype=bool)
    is_img[master_occ] = False
    imgs = occ_order[is_img[occ_order]]
    node_id[imgs] = np.arange(nv + 1, nv + 1 + len(imgs))
    nodes = np.empty((len(first), 3))
    nodes[node_id - 1] = occ_pos
    elem_nodes = node_id[inv].reshape(ne, 4)
    attr = np.asarray(mesh.attr, dtype=np.int64)
    with open(path, "w") as f:
        f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n")
        f.write(f"$Nodes\n{len(nodes)}\n")
        f.write("".join(f"{i + 1} {x:.17g} {y:.17g} {z:.17g}\n"
                        for i, (x, y, z) in enumerate(nodes)))
        f.write("$EndNodes\n")
        f.write(f"$Elements\n{ne}\n")
        f.write("".join(f"{e + 1} {TET} 2 {a} {a} {n[0]} {n[1]} {n[2]} {n[3]}\n"
                        for e, (a, n) in enumerate(zip(attr, elem_nodes))))
        f.write("$EndElements\n")
        if len(imgs):
            f.write("$Periodic\n1\n2 2 1\n")
            f.write(f"{len(imgs)}\n")
            masters = node_id[master_occ[occ_vertex[imgs]]]
            f.write("".join(f"{s} {m}\n" for s, m in zip(node_id[imgs], masters)))
            f.write("$EndPeriodic\n")
