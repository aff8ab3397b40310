"""Synthetic box meshes of linear tetrahedra (stand-in for the gmsh reader, ReadGMSH.f90).

An nx x ny x nz grid of hexahedra, each split into 6 positively oriented tetrahedra along its
main diagonal (Kuhn split).  Conventions follow the reference's mesh tapes:
  * nodes lexicographic, x fastest;
  * elements hex-lexicographic, then the fixed 6-tet order below;
  * local faces in gmsh order {0,1,2}, {0,1,3}, {0,2,3}, {1,2,3} (gmshprocessing.py:32-42);
  * neighbours across each local face found by matching sorted node triples
    (gmshprocessing.py:258-288); -1 marks a boundary face.
The node order of every tet gives a positive Jacobian determinant, which the reference's
mass-eliminated matrices require (FiniteElementAnalysis.f90:245).
"""
from dataclasses import dataclass, field

import numpy as np

F2K = np.array([[0, 1, 2], [0, 1, 3], [0, 2, 3], [1, 2, 3]])
_PERMS = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]


def _perm_sign(p):
    s = 1
    p = list(p)
    for i in range(3):
        for j in range(i + 1, 3):
            if p[i] > p[j]:
                s = -s
    return s


@dataclass
class Mesh:
    rg: np.ndarray          # [NN, 3]
    node: np.ndarray        # [NE, 4] int32
    neighbors: np.ndarray   # [NE, 4] int32, -1 on the boundary
    mat: np.ndarray         # [NE] int32
    Nm: int
    shape: tuple = field(default=())

    @property
    def NE(self):
        return int(self.node.shape[0])

    @property
    def NN(self):
        return int(self.rg.shape[0])

    @property
    def NENK(self):
        return 4 * self.NE

    def node_coords(self):
        """Coordinates of every DG node, [NENK, 3] (element-major, gmsh local order)."""
        return self.rg[self.node.reshape(-1)]

    def centroids(self):
        return self.rg[self.node].mean(axis=1)


def neighbours(node):
    """Element across each local face (-1 on the boundary) by sorted node-triple matching."""
    NE = node.shape[0]
    faces = np.sort(node[:, F2K], axis=2).reshape(-1, 3).astype(np.int64)    # [4NE, 3]
    key = (faces[:, 0] << 42) | (faces[:, 1] << 21) | faces[:, 2]
    order = np.argsort(key, kind="stable")
    ks = key[order]
    nb = np.full(4 * NE, -1, dtype=np.int64)
    same = ks[1:] == ks[:-1]
    a = order[:-1][same]
    b = order[1:][same]
    nb[a] = b // 4
    nb[b] = a // 4
    return nb.reshape(NE, 4).astype(np.int32)


def box_mesh(nx, ny, nz, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), material=None, Nm=1):
    """Box [lo, hi] split into nx*ny*nz hexes x 6 tets.

    material: optional callable(centroids [NE,3]) -> int array of material ids.
    """
    lo = np.asarray(lo, dtype=np.float64)
    hi = np.asarray(hi, dtype=np.float64)
    xs = lo[0] + (hi[0] - lo[0]) * np.arange(nx + 1) / nx
    ys = lo[1] + (hi[1] - lo[1]) * np.arange(ny + 1) / ny
    zs = lo[2] + (hi[2] - lo[2]) * np.arange(nz + 1) / nz
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    rg = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)

    def nid(i, j, k):
        return i + (nx + 1) * (j + (ny + 1) * k)

    k3, j3, i3 = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    i3, j3, k3 = i3.ravel(), j3.ravel(), k3.ravel()
    tets = []
    for p in _PERMS:
        e = [np.zeros(3, dtype=int) for _ in range(3)]
        e[0][p[0]] = 1
        e[1][p[1]] = 1
        e[2][p[2]] = 1
        v0 = (0, 0, 0)
        v1 = tuple(e[0])
        v2 = tuple(e[0] + e[1])
        v3 = (1, 1, 1)
        verts = [v0, v1, v2, v3] if _perm_sign(p) > 0 else [v0, v2, v1, v3]
        tets.append(np.stack([nid(i3 + v[0], j3 + v[1], k3 + v[2]) for v in verts], axis=1))
    node = np.stack(tets, axis=1).reshape(-1, 4).astype(np.int32)      # hex-major, 6 tets per hex
    nb = neighbours(node)
    if material is None:
        mat = np.zeros(node.shape[0], dtype=np.int32)
    else:
        mat = np.asarray(material(rg[node].mean(axis=1)), dtype=np.int32)
    return Mesh(rg=rg, node=node, neighbors=nb, mat=mat, Nm=int(Nm), shape=(nx, ny, nz))
