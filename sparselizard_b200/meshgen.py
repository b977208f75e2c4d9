"""Seeded synthetic meshes written as GMSH v2 ASCII ``.msh`` files.

sparselizard's native reader (src/io/gmsh/gmshinterface.cpp:157-298) accepts
GMSH format < 4, takes the first element tag as the physical region, and
numbers nodes in file order.  Every mesh here is a structured grid on the unit
square / cube whose interior nodes are jittered uniformly by +-``jitter``*h
with numpy's PCG64 generator, so a (shape, seed) pair always produces the same
file and therefore the same DOF numbering in sparselizard.

GMSH element type numbers used: 1 line2, 2 tri3, 3 quad4, 4 tet4, 5 hex8.
"""
from __future__ import annotations

import numpy as np

# Physical region numbers shared by the drivers (sparselizard keeps one
# numbering space per element dimension).
VOL = 1          # all volume (3D) or surface (2D) elements
BOUNDARY = 2     # whole boundary (2D: lines, 3D: faces)
CLAMP = 3        # 3D: the z = 0 face
ORDER_REGION_BASE = 10   # p-adaptive meshes: region 10+p holds the order-p elements
MATERIAL_REGION_BASE = 20  # material regions 20..23


def _grid_nodes(shape, jitter, rng):
    axes = [np.linspace(0.0, 1.0, n + 1) for n in shape]
    mesh = np.meshgrid(*axes, indexing="ij")
    pts = np.stack([m.ravel(order="F") for m in mesh], axis=1)  # x fastest
    h = np.array([1.0 / n for n in shape])
    interior = np.ones(pts.shape[0], dtype=bool)
    for d in range(len(shape)):
        interior &= (pts[:, d] > 1e-12) & (pts[:, d] < 1 - 1e-12)
    noise = rng.uniform(-jitter, jitter, size=pts.shape) * h
    pts[interior] += noise[interior]
    if pts.shape[1] == 2:
        pts = np.concatenate([pts, np.zeros((pts.shape[0], 1))], axis=1)
    return pts


def _write(path, nodes, blocks):
    """blocks: list of (gmsh_type, physical_tags[n], connectivity[n, k]) (0-based nodes)."""
    nel = sum(b[2].shape[0] for b in blocks)
    with open(path, "w") as f:
        f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n")
        f.write(f"$Nodes\n{nodes.shape[0]}\n")
        ids = np.arange(1, nodes.shape[0] + 1)
        np.savetxt(f, np.column_stack([ids, nodes]), fmt=["%d", "%.17g", "%.17g", "%.17g"])
        f.write("$EndNodes\n")
        f.write(f"$Elements\n{nel}\n")
        eid = 1
        for gtype, tags, conn in blocks:
            n = conn.shape[0]
            cols = [np.arange(eid, eid + n), np.full(n, gtype), np.full(n, 2), tags, tags, conn + 1]
            arr = np.column_stack(cols).astype(np.int64)
            np.savetxt(f, arr, fmt="%d")
            eid += n
        f.write("$EndElements\n")


def quad_mesh(path, n, jitter=0.2, seed=1):
    """n x n quadrangles on the unit square; VOL = all quads, BOUNDARY = boundary lines."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nodes = _grid_nodes((n, n), jitter, rng)
    nid = lambda i, j: i + (n + 1) * j
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    i, j = i.ravel(order="F"), j.ravel(order="F")
    quads = np.stack([nid(i, j), nid(i + 1, j), nid(i + 1, j + 1), nid(i, j + 1)], axis=1)
    k = np.arange(n)
    lines = np.concatenate([
        np.stack([nid(k, 0), nid(k + 1, 0)], axis=1),
        np.stack([nid(n, k), nid(n, k + 1)], axis=1),
        np.stack([nid(k + 1, n), nid(k, n)], axis=1),
        np.stack([nid(0, k + 1), nid(0, k)], axis=1),
    ])
    _write(path, nodes, [
        (3, np.full(quads.shape[0], VOL), quads),
        (1, np.full(lines.shape[0], BOUNDARY), lines),
    ])
    return {"nelem": quads.shape[0], "nnodes": nodes.shape[0]}


def tri_mesh(path, n, jitter=0.2, seed=1):
    """n x n squares split into 2 triangles each (diagonal (i,j)-(i+1,j+1));
    VOL = all triangles, BOUNDARY = boundary lines."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nodes = _grid_nodes((n, n), jitter, rng)
    nid = lambda i, j: i + (n + 1) * j
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    i, j = i.ravel(order="F"), j.ravel(order="F")
    a, b, c, d = nid(i, j), nid(i + 1, j), nid(i + 1, j + 1), nid(i, j + 1)
    tris = np.concatenate([np.stack([a, b, c], axis=1), np.stack([a, c, d], axis=1)])
    k = np.arange(n)
    lines = np.concatenate([
        np.stack([nid(k, 0), nid(k + 1, 0)], axis=1),
        np.stack([nid(n, k), nid(n, k + 1)], axis=1),
        np.stack([nid(k + 1, n), nid(k, n)], axis=1),
        np.stack([nid(0, k + 1), nid(0, k)], axis=1),
    ])
    _write(path, nodes, [
        (2, np.full(tris.shape[0], VOL), tris),
        (1, np.full(lines.shape[0], BOUNDARY), lines),
    ])
    return {"nelem": tris.shape[0], "nnodes": nodes.shape[0]}


def _hex_conn(n):
    nid = lambda i, j, k: i + (n + 1) * (j + (n + 1) * k)
    i, j, k = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    i, j, k = i.ravel(order="F"), j.ravel(order="F"), k.ravel(order="F")
    hexes = np.stack([nid(i, j, k), nid(i + 1, j, k), nid(i + 1, j + 1, k), nid(i, j + 1, k),
                      nid(i, j, k + 1), nid(i + 1, j, k + 1), nid(i + 1, j + 1, k + 1), nid(i, j + 1, k + 1)], axis=1)
    return hexes, nid


def _bottom_quads(n, nid):
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    i, j = i.ravel(order="F"), j.ravel(order="F")
    return np.stack([nid(i, j, 0), nid(i, j + 1, 0), nid(i + 1, j + 1, 0), nid(i + 1, j, 0)], axis=1)


def hex_mesh(path, n, jitter=0.15, seed=1):
    """n^3 hexahedra on the unit cube; VOL = all hexes, CLAMP = quads of the z = 0 face."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nodes = _grid_nodes((n, n, n), jitter, rng)
    hexes, nid = _hex_conn(n)
    bottom = _bottom_quads(n, nid)
    _write(path, nodes, [
        (5, np.full(hexes.shape[0], VOL), hexes),
        (3, np.full(bottom.shape[0], CLAMP), bottom),
    ])
    return {"nelem": hexes.shape[0], "nnodes": nodes.shape[0]}


# Kuhn split of the unit cube into 6 tets sharing the main diagonal 0-6; the
# local hex numbering is the one of _hex_conn.  Consistent diagonals across
# neighbouring cubes make the tet mesh conforming.
_KUHN = np.array([[0, 1, 2, 6], [0, 2, 3, 6], [0, 3, 7, 6], [0, 7, 4, 6], [0, 4, 5, 6], [0, 5, 1, 6]])


def tet_mesh(path, n, jitter=0.1, seed=1, element_tags=None):
    """n^3 cubes split into 6 tets each.  element_tags (len 6 n^3) gives each tet's
    physical region; default VOL for all.  Also writes the CLAMP face triangles."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nodes = _grid_nodes((n, n, n), jitter, rng)
    hexes, nid = _hex_conn(n)
    tets = hexes[:, _KUHN].reshape(-1, 4)
    # Orient every tet positively (sparselizard takes |detJ| anyway).
    p = nodes[tets]
    vol = np.einsum("ij,ij->i", np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), p[:, 3] - p[:, 0])
    neg = vol < 0
    tets[neg] = tets[neg][:, [0, 2, 1, 3]]
    tags = np.full(tets.shape[0], VOL) if element_tags is None else np.asarray(element_tags)
    bottom = _bottom_quads(n, nid)
    tris = np.concatenate([bottom[:, [0, 1, 2]], bottom[:, [0, 2, 3]]])
    _write(path, nodes, [
        (4, tags, tets),
        (2, np.full(tris.shape[0], CLAMP), tris),
    ])
    return {"nelem": tets.shape[0], "nnodes": nodes.shape[0]}


def workload_mesh(kind, n, path):
    """The seeded mesh of one benchmark workload at size n:
    "quad"       n x n q4, jitter 0.2h (Poisson);
    "hex"        n^3 hexahedra, jitter 0.15h (elasticity, z = 0 face clamped);
    "tet_orders" n^3 x 6 tets, jitter 0.1h, each tet in region
                 ORDER_REGION_BASE + p with p uniform in 1..5 (p-adaptive Helmholtz);
    "tet_sigma"  n^3 x 6 tets, jitter 0.1h, each tet in one of the 4 material
                 regions MATERIAL_REGION_BASE + 0..3 (eddy currents)."""
    if kind == "quad":
        return quad_mesh(path, n, jitter=0.2, seed=1)
    if kind == "hex":
        return hex_mesh(path, n, jitter=0.15, seed=1)
    if kind == "tet_orders":
        rng = np.random.Generator(np.random.PCG64(1))
        tags = ORDER_REGION_BASE + rng.integers(1, 6, size=6 * n ** 3)
        return tet_mesh(path, n, jitter=0.1, seed=1, element_tags=tags)
    if kind == "tet_sigma":
        rng = np.random.Generator(np.random.PCG64(1))
        tags = MATERIAL_REGION_BASE + rng.integers(0, 4, size=6 * n ** 3)
        return tet_mesh(path, n, jitter=0.1, seed=1, element_tags=tags)
    raise ValueError(kind)
