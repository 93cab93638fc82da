"""Renumbering of a mesh for the general-mesh tests: the same cells, nodes and ghosts
under other ids, and each cell's faces starting at another corner."""
import dataclasses

import numpy as np


def permute_mesh(mesh, seed=0, rotate=True):
    """Random cell and node ids (default_rng(seed)) and, with ``rotate``, a random cyclic
    shift of every cell's local node order (its NC and its ghosts' NSIDE follow).  Ghost
    ids and the bc.in line order are kept.  Returns (mesh, cell_perm) where new cell id
    cell_perm[c] + 1 holds old cell c + 1."""
    rng = np.random.default_rng(seed)
    ne, nn = mesh.neles, mesh.nods
    cperm = rng.permutation(ne)          # old cell c -> new index cperm[c]
    nperm = rng.permutation(nn)          # old node n -> new index nperm[n]
    rot = rng.integers(0, 4, ne) if rotate else np.zeros(ne, int)
    inv = np.argsort(cperm)
    nod = np.zeros_like(mesh.nod)
    nc = np.zeros_like(mesh.nc)
    for new in range(ne):
        c, r = inv[new], rot[inv[new]]
        for k in range(4):
            nod[new, k] = nperm[mesh.nod[c, (k + r) % 4] - 1] + 1
            v = mesh.nc[c, (k + r) % 4]
            nc[new, k] = cperm[v - 1] + 1 if v <= ne else v
    x = np.zeros(nn)
    y = np.zeros(nn)
    x[nperm] = mesh.x
    y[nperm] = mesh.y
    xm = ym = None
    if mesh.x_mm is not None:
        xm = np.zeros(nn)
        ym = np.zeros(nn)
        xm[nperm] = mesh.x_mm
        ym[nperm] = mesh.y_mm
    par = mesh.nparent - 1
    side = ((mesh.nside - 1 - rot[par]) % 4 + 1).astype(np.int32)
    out = dataclasses.replace(mesh, x=x, y=y, x_mm=xm, y_mm=ym, nod=nod.astype(np.int32),
                              nc=nc.astype(np.int32), nparent=(cperm[par] + 1).astype(np.int32),
                              nside=side, shape=None)
    return out, cperm
