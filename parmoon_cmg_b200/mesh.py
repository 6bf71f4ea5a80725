"""Structured quadrilateral / hexahedral meshes and their Q1/Q2 DOF maps.

This plays the role of ParMooN's TDomain refinement plus TFESpace2D/3D
construction for the unit square / cube (the reference builds these on the
host too; they are inputs of the hot path, not part of it).  The arrays have
the reference's layout: cell vertices counter-clockwise (3D: bottom face then
top face), local DOFs in the tensor-product order of the basis functions
(x fastest), global DOFs ordered [inner | Dirichlet] with the whole boundary
Dirichlet, BeginIndex stepping by the number of basis functions.

The numbering inside each class is lexicographic, which differs from the
reference's refinement-tree order; callers that need the reference's own
numbering pass its arrays to the library instead (the library never renumbers).
"""
import numpy as np


def structured_space(dim, order, n, lo=0.0, hi=1.0):
    """Uniform n^dim mesh of [lo,hi]^dim with Q_order elements."""
    p = order
    m = p * n + 1  # grid nodes per direction
    h = (hi - lo) / n
    nc = n ** dim
    # cell multi-indices, x fastest (cell c = i + n*j + n*n*k)
    idx = np.indices((n,) * dim).reshape(dim, -1)[::-1]  # idx[0]=i (x) fastest
    # vertices
    if dim == 2:
        off = np.array([[0, 0], [1, 0], [1, 1], [0, 1]])
    else:
        off = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                        [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]])
    verts = (idx.T[:, None, :] + off[None, :, :]) * h + lo  # nc x nv x dim
    # local DOF offsets in tensor order (x fastest)
    loc = np.indices((p + 1,) * dim).reshape(dim, -1)[::-1].T  # nbf x dim
    node = p * idx.T[:, None, :] + loc[None, :, :]  # nc x nbf x dim grid indices
    lin = node[..., 0] + m * node[..., 1] + (m * m * node[..., 2] if dim == 3 else 0)
    # classify grid nodes: boundary = any index 0 or m-1
    g = np.indices((m,) * dim).reshape(dim, -1)[::-1]
    bnd = np.zeros(m ** dim, bool)
    for a in range(dim):
        bnd |= (g[a] == 0) | (g[a] == m - 1)
    inner = np.flatnonzero(~bnd)
    dirich = np.flatnonzero(bnd)
    new = np.empty(m ** dim, np.int64)
    new[inner] = np.arange(len(inner))
    new[dirich] = len(inner) + np.arange(len(dirich))
    gn = new[lin].astype(np.int32).reshape(-1)
    nbf = (p + 1) ** dim
    return {
        "dim": dim, "order": order, "n": n,
        "coords": np.ascontiguousarray(verts.reshape(-1), np.float64),
        "global_numbers": gn,
        "begin_index": (np.arange(nc + 1) * nbf).astype(np.int32),
        "n_dof": m ** dim, "n_active": len(inner), "n_cells": nc,
    }


def parent_map(dim, n_fine):
    """Parent cell of every cell of a uniform n_fine^dim mesh in the n_fine/2 mesh."""
    idx = np.indices((n_fine,) * dim).reshape(dim, -1)[::-1] // 2
    nc = n_fine // 2
    par = idx[0] + nc * idx[1] + (nc * nc * idx[2] if dim == 3 else 0)
    return par.astype(np.int32)


def structured_hierarchy(dim, order, n_coarse, n_levels):
    """Spaces of uniform refinements n_coarse * 2^l, coarsest first, with parent maps."""
    spaces, parents = [], [None]
    for l in range(n_levels):
        n = n_coarse * 2 ** l
        spaces.append(structured_space(dim, order, n))
        if l > 0:
            parents.append(parent_map(dim, n))
    return spaces, parents


def dof_coords(space):
    """Physical coordinates of every DOF (n_dof x dim)."""
    dim, p = space["dim"], space["order"]
    nbf = (p + 1) ** dim
    verts = space["coords"].reshape(-1, 2 ** dim, dim)
    loc = np.indices((p + 1,) * dim).reshape(dim, -1)[::-1].T / p  # in [0,1]
    v0 = verts[:, 0, :]
    if dim == 2:
        e = np.stack([verts[:, 1] - v0, verts[:, 3] - v0], 1)
    else:
        e = np.stack([verts[:, 1] - v0, verts[:, 3] - v0, verts[:, 4] - v0], 1)
    pts = v0[:, None, :] + np.einsum("ka,cad->ckd", loc, e)
    out = np.zeros((space["n_dof"], dim))
    out[space["global_numbers"].reshape(-1, nbf)] = pts
    return out
