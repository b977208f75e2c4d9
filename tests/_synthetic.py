"""Seeded synthetic element groups for C-ABI level tests (no sparselizard).

A structured grid of bilinear quadrangles (or trilinear hexahedra) gives
well-conditioned Jacobians; form-function tables, coefficient data and
addresses are random but reproducible.
"""
from __future__ import annotations

import numpy as np

from sparselizard_b200 import abi


def gauss_1d(n):
    x, w = np.polynomial.legendre.leggauss(n)
    return x, w


def lagrange_q4(gp):
    """[1+2][4][ngp]: values then d/dki, d/deta of bilinear functions on [-1,1]^2."""
    k, e = gp[:, 0], gp[:, 1]
    sk = np.array([-1, 1, 1, -1.0])
    se = np.array([-1, -1, 1, 1.0])
    val = 0.25 * (1 + np.outer(sk, k)) * (1 + np.outer(se, e))
    dk = 0.25 * sk[:, None] * (1 + np.outer(se, e))
    de = 0.25 * (1 + np.outer(sk, k)) * se[:, None]
    return np.stack([val, dk, de])


def quad_mesh_arrays(n, rng, jitter=0.2):
    xs = np.linspace(0, 1, n + 1)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    pts = np.stack([X.ravel(order="F"), Y.ravel(order="F"), np.zeros(X.size)], axis=1)
    inner = (pts[:, 0] > 0) & (pts[:, 0] < 1) & (pts[:, 1] > 0) & (pts[:, 1] < 1)
    pts[inner, :2] += rng.uniform(-jitter, jitter, (inner.sum(), 2)) / n
    nid = lambda i, j: i + (n + 1) * j
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    i, j = i.ravel(order="F"), j.ravel(order="F")
    conn = np.stack([nid(i, j), nid(i + 1, j), nid(i + 1, j + 1), nid(i, j + 1)], axis=1).astype(np.int32)
    return pts.ravel(), conn.ravel()


def group(rng, nelem_grid=8, ntf=5, ndof=3, nterms=3, ngp1=3, norient=2, ndests=2, ndofs=60, rhs=False, p_neg=0.1,
          with_elemdata=True, symmetric=False):
    """Returns (GroupBuilder, xyz, conn, extra) for a random quad group.

    symmetric: element matrices symmetric by construction (ntf == ndof).
    Terms 2k and 2k+1 are mirrors: each one's dof table is a copy of the
    other's test-function table, and their coefficients are the same
    expression with the operands of one product swapped; equal scales.  An
    odd last term is its own mirror."""
    if symmetric:
        assert ntf == ndof and not rhs
    xyz, conn = quad_mesh_arrays(nelem_grid, rng)
    nelem = nelem_grid * nelem_grid
    x, w = gauss_1d(ngp1)
    gp = np.array([[a, b] for b in x for a in x])
    weights = np.array([wa * wb for wb in w for wa in x * 0 + w])
    ngp = gp.shape[0]
    lag = lagrange_q4(gp)
    elems = rng.permutation(nelem).astype(np.int32)
    orient = np.sort(rng.integers(0, norient, nelem)).astype(np.int32)
    tables = [rng.standard_normal((norient, ntf, ngp)) for _ in range(nterms)]
    mirror = [t ^ 1 if (t ^ 1) < nterms else t for t in range(nterms)]
    if symmetric:
        tables += [tables[mirror[t]].copy() for t in range(nterms)]
    elif not rhs:
        tables += [rng.standard_normal((norient, ndof, ngp)) for _ in range(nterms)]
    consts = rng.standard_normal(4)
    # coef_t = c0*invJ(0,t%2)*invJ(1,(t+1)%2) + c1*E/(detJ) + x coordinate, E per element.
    nodes = [
        (abi.OP_CONST, 0, 0, 0),       # 0 c0
        (abi.OP_CONST, 1, 0, 0),       # 1 c1
        (abi.OP_DETJAC, 0, 0, 0),      # 2
        (abi.OP_INV, 2, 0, 0),         # 3 1/detJ
        (abi.OP_COORD, 0, 0, 0),       # 4 x
    ]
    if with_elemdata:
        nodes.append((abi.OP_ELEM, 0, 0, 0))  # 5 E
    else:
        nodes.append((abi.OP_CONST, 2, 0, 0))
    base = len(nodes)
    coef_nodes = []
    for t in range(nterms):
        k = t // 2 if symmetric else t
        a, b = k % 2, (k + 1) % 2
        nodes.append((abi.OP_INVJAC, 0, a, 0))
        i1 = len(nodes) - 1
        nodes.append((abi.OP_INVJAC, 1, b, 0))
        i2 = len(nodes) - 1
        nodes.append((abi.OP_MUL, i2, i1, 0) if symmetric and t % 2 else (abi.OP_MUL, i1, i2, 0))
        m = len(nodes) - 1
        nodes.append((abi.OP_MUL, m, 0, 0))
        m0 = len(nodes) - 1
        nodes.append((abi.OP_MUL, 5, 3, 0))
        e1 = len(nodes) - 1
        nodes.append((abi.OP_MUL, e1, 1, 0))
        e2 = len(nodes) - 1
        nodes.append((abi.OP_ADD, m0, e2, 0))
        s = len(nodes) - 1
        nodes.append((abi.OP_ADD, s, 4, 0))
        coef_nodes.append(len(nodes) - 1)
    terms = []
    scales = [float(rng.choice([1.0, -0.5, 2.0])) for _ in range(nterms)]
    for t in range(nterms):
        terms.append((t, -1 if rhs else nterms + t, coef_nodes[t], scales[min(t, mirror[t])] if symmetric else scales[t]))

    def addr(rows):
        a = rng.integers(0, ndofs, (rows, nelem)).astype(np.int32)
        a[rng.random((rows, nelem)) < p_neg] = -1
        return a

    dests = []
    for d in range(ndests):
        dests.append((addr(ntf), None if rhs else addr(ndof), float(rng.choice([1.0, 3.0, -2.5]))))
    elemdata = [rng.lognormal(0, 0.5, nelem)] if with_elemdata else []
    gb = abi.GroupBuilder(elemtype=3, dim=2, elems=elems, orient=orient, norient=norient, weights=weights,
                          lagrange=lag, ncurvednodes=4, ntf=ntf, ndof=1 if rhs else ndof, tables=tables, nodes=nodes,
                          consts=consts, terms=terms, dests=dests, elemdata=elemdata)
    return gb, xyz, conn
