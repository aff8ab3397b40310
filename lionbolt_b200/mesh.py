"""Meshes of linear tetrahedra: the gmsh MSH 4.1 ASCII reader (ReadGMSH.f90 with gmshprocessing.py)
and synthetic box meshes.

A box mesh is an nx x ny x nz grid of hexahedra, each split into 6 positively oriented tetrahedra
along its main diagonal (Kuhn split).  Conventions follow the reference's mesh tapes:
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
    """Element across each local face (-1 on the boundary) by sorted node-triple matching
    (gmshprocessing.py:258-288).  A face shared by more than two elements is an error."""
    NE = node.shape[0]
    faces = np.sort(node[:, F2K], axis=2).reshape(-1, 3).astype(np.int64)    # [4NE, 3]
    order = np.lexsort((faces[:, 2], faces[:, 1], faces[:, 0]))
    fs = faces[order]
    same = np.all(fs[1:] == fs[:-1], axis=1)
    if np.any(same[1:] & same[:-1]):
        raise ValueError("mesh: a face is shared by more than two elements")
    nb = np.full(4 * NE, -1, dtype=np.int64)
    a = order[:-1][same]
    b = order[1:][same]
    nb[a] = b // 4
    nb[b] = a // 4
    return nb.reshape(NE, 4).astype(np.int32)


def _sections(path):
    """{name: [lines]} of the $Name ... $EndName sections of an MSH file."""
    out, name, buf = {}, None, []
    with open(path) as f:
        for raw in f:
            line = raw.strip()
            if name is None:
                if line.startswith("$") and not line.startswith("$End"):
                    name, buf = line[1:], []
            elif line == "$End" + name:
                out[name] = buf
                name = None
            else:
                buf.append(line)
    return out


def read_gmsh(path):
    """Tetrahedral mesh from a gmsh MSH 4.1 ASCII file, as the reference reads it (ReadGMSH.f90:3-236
    with gmshprocessing.py): the nodes of $Nodes (indexed by tag); the 3-D elements of $Elements in
    block order (4-node tetrahedra only); the material of an element = the physical tag of its volume
    entity in $Entities (a volume without a physical tag is material 1, ReadGMSH.f90:119-139; a
    volume with more than one tag, or untagged volumes next to a tag other than 1, is an error);
    neighbours by face matching.  Physical tags are
    1-based in the file and 0-based in the returned mesh, and must not skip numbers."""
    sec = _sections(path)
    fmt = sec.get("MeshFormat", [""])[0].split()
    if len(fmt) < 2 or not fmt[0].startswith("4.1") or fmt[1] != "0":
        raise ValueError(f"{path}: only gmsh MSH 4.1 ASCII files are read (found {' '.join(fmt)!r})")
    # volume entities and their physical tags
    ent = sec.get("Entities")
    if not ent:
        raise ValueError(f"{path}: no $Entities section")
    npts, ncur, nsur, nvol = (int(v) for v in ent[0].split()[:4])
    vol_mat, untagged = {}, False
    for line in ent[1 + npts + ncur + nsur:1 + npts + ncur + nsur + nvol]:
        tok = line.split()
        ntags = int(tok[7])
        if ntags > 1:
            raise ValueError(f"{path}: volume {tok[0]} has {ntags} physical tags; a volume takes one material")
        # a volume without a physical tag is material 1 (homogeneous transport)
        vol_mat[int(tok[0])] = int(tok[8]) if ntags == 1 else 1
        untagged = untagged or ntags == 0
    # untagged volumes are accepted next to volumes tagged 1, not next to other materials
    if untagged and any(t != 1 for t in vol_mat.values()):
        raise ValueError(f"{path}: materials are given for some volumes but not for all")
    # nodes: blocks of (entityDim entityTag parametric n), n tags, n coordinate lines
    nd = sec["Nodes"]
    nblocks, nnodes = (int(v) for v in nd[0].split()[:2])
    tags, coords, i = [], [], 1
    for _ in range(nblocks):
        _dim, _etag, param, n = (int(v) for v in nd[i].split())
        if param != 0:
            raise ValueError(f"{path}: parametric node coordinates are not supported")
        tags.extend(int(v) for v in nd[i + 1:i + 1 + n])
        coords.extend(nd[i + 1 + n:i + 1 + 2 * n])
        i += 1 + 2 * n
    if len(tags) != nnodes:
        raise ValueError(f"{path}: $Nodes lists {len(tags)} nodes, its header {nnodes}")
    rg = np.array([[float(v) for v in c.split()[:3]] for c in coords], dtype=np.float64)
    tag_to_idx = np.full(max(tags) + 1, -1, dtype=np.int64)
    tag_to_idx[np.array(tags)] = np.arange(len(tags))
    # elements: blocks of (entityDim entityTag elementType n), n lines "tag node..."
    el = sec["Elements"]
    nblocks = int(el[0].split()[0])
    nodes, mats, i = [], [], 1
    for _ in range(nblocks):
        dim, etag, etype, n = (int(v) for v in el[i].split())
        rows = el[i + 1:i + 1 + n]
        i += 1 + n
        if dim != 3:
            continue
        if etype != 4:
            raise ValueError(f"{path}: element type {etype} in volume {etag}; only 4-node tetrahedra are supported")
        blk = np.array([[int(v) for v in r.split()[1:5]] for r in rows], dtype=np.int64)
        nodes.append(tag_to_idx[blk])
        mats.append(np.full(n, vol_mat.get(etag, 1) - 1, dtype=np.int32))
    if not nodes:
        raise ValueError(f"{path}: no tetrahedra")
    node = np.concatenate(nodes).astype(np.int32)
    if np.any(node < 0):
        raise ValueError(f"{path}: an element references an unknown node tag")
    mat = np.concatenate(mats)
    Nm = int(mat.max()) + 1
    if set(np.unique(mat).tolist()) != set(range(Nm)):
        raise ValueError(f"{path}: the physical (material) tags skip numbers")
    return Mesh(rg=rg, node=node, neighbors=neighbours(node), mat=mat, Nm=Nm)


def write_gmsh(mesh, path):
    """Writes a mesh as gmsh MSH 4.1 ASCII: one volume entity per material (physical tag = material
    + 1), nodes tagged 1..NN, tetrahedra tagged 1..NE in element order, so read_gmsh returns the same
    mesh when its elements are grouped by material in increasing order."""
    NN, NE = mesh.NN, mesh.NE
    lo, hi = mesh.rg.min(axis=0), mesh.rg.max(axis=0)
    with open(path, "w") as f:
        f.write("$MeshFormat\n4.1 0 8\n$EndMeshFormat\n")
        f.write(f"$Entities\n0 0 0 {mesh.Nm}\n")
        for m in range(mesh.Nm):
            f.write(f"{m + 1} {lo[0]!r} {lo[1]!r} {lo[2]!r} {hi[0]!r} {hi[1]!r} {hi[2]!r} 1 {m + 1} 0\n")
        f.write("$EndEntities\n")
        f.write(f"$Nodes\n1 {NN} 1 {NN}\n3 1 0 {NN}\n")
        f.write("".join(f"{k + 1}\n" for k in range(NN)))
        f.write("".join(f"{x!r} {y!r} {z!r}\n" for x, y, z in mesh.rg.tolist()))
        f.write("$EndNodes\n")
        f.write(f"$Elements\n{mesh.Nm} {NE} 1 {NE}\n")
        for m in range(mesh.Nm):
            idx = np.nonzero(mesh.mat == m)[0]
            f.write(f"3 {m + 1} 4 {idx.size}\n")
            f.write("".join(f"{e + 1} {a + 1} {b + 1} {c + 1} {d + 1}\n" for e, (a, b, c, d) in zip(idx.tolist(), mesh.node[idx].tolist())))
        f.write("$EndElements\n")


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
