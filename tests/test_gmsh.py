"""gmsh MSH 4.1 ASCII reader (ReadGMSH.f90 with gmshprocessing.py): round trips through the writer,
the reference's own mesh files where its tree is present, and the errors the reference reports."""
import os

import numpy as np
import pytest

from helpers import jittered
from lionbolt_b200 import _lib
from lionbolt_b200 import mesh as M
from lionbolt_b200 import problems as P
from test_host import HostHandle

# root of a Lionbolt source tree (its shipped meshes are read where it is given)
REF = os.environ.get("LIONBOLT_REFERENCE")


def _grouped(m):
    """The mesh's elements grouped by material (the order write_gmsh stores them in)."""
    return np.concatenate([np.nonzero(m.mat == g)[0] for g in range(m.Nm)])


@pytest.mark.parametrize("which", ["two_material", "jittered"])
def test_round_trip(tmp_path, which):
    m = P.config1_small(n=(4, 4, 8)).mesh if which == "two_material" else \
        jittered(M.box_mesh(5, 4, 3, (0, 0, 0), (2.5, 2.0, 1.5)), 0.06)
    path = str(tmp_path / "m.msh")
    M.write_gmsh(m, path)
    r = M.read_gmsh(path)
    order = _grouped(m)
    assert r.Nm == m.Nm and r.NE == m.NE and r.NN == m.NN
    assert np.array_equal(r.rg, m.rg)
    assert np.array_equal(r.node, m.node[order])
    assert np.array_equal(r.mat, m.mat[order])
    # neighbours: the same elements across the same local faces, in the new numbering
    new_of_old = np.empty(m.NE, np.int64)
    new_of_old[order] = np.arange(m.NE)
    expect = np.where(m.neighbors[order] >= 0, new_of_old[np.maximum(m.neighbors[order], 0)], -1)
    assert np.array_equal(r.neighbors, expect)


@pytest.mark.parametrize("rel, ne, nn, counts", [
    ("validation/operators/simple_cube.msh", 12741, 2786, [12741]),
    ("examples/water_tank_with_aluminum/het_cube_spherical_beam.msh", 78771, 13707, [63313, 15458]),
])
def test_reference_meshes(rel, ne, nn, counts):
    if not REF or not os.path.exists(os.path.join(REF, rel)):
        pytest.skip("LIONBOLT_REFERENCE does not name a Lionbolt tree with its mesh files")
    path = os.path.join(REF, rel)
    m = M.read_gmsh(path)
    assert (m.NE, m.NN) == (ne, nn)
    assert np.bincount(m.mat).tolist() == counts
    # every interior face is shared both ways, and the mesh is closed (boundary faces pair up)
    e, f = np.nonzero(m.neighbors >= 0)
    ep = m.neighbors[e, f]
    assert np.all(np.any(m.neighbors[ep] == e[:, None], axis=1))
    hh = HostHandle()
    assert hh.mesh(m) == 0, hh.error()
    assert hh.quad(*P.quadrature(2, 4)) == 0, hh.error()   # a cyclic mesh would be reported here
    n = np.zeros(1, np.int32)
    assert hh.lib.lb_mesh_types(hh.h, _lib.iptr(n)) == 0 and n[0] == 0   # general shapes: 64-byte records


def _write(tmp_path, text):
    p = tmp_path / "bad.msh"
    p.write_text(text)
    return str(p)


ONE_TET = """$MeshFormat
4.1 0 8
$EndMeshFormat
$Entities
0 0 0 1
1 0 0 0 1 1 1 {tags} 0
$EndEntities
$Nodes
1 4 1 4
3 1 0 4
1
2
3
4
0 0 0
1 0 0
0 1 0
0 0 1
$EndNodes
$Elements
1 1 1 1
3 1 {etype} 1
1 1 2 3 4{extra}
$EndElements
"""


def test_errors(tmp_path):
    ok = M.read_gmsh(_write(tmp_path, ONE_TET.format(tags="1 1", etype=4, extra="")))
    assert ok.NE == 1 and ok.Nm == 1 and np.all(ok.neighbors == -1)
    with pytest.raises(ValueError, match="only 4-node tetrahedra"):
        M.read_gmsh(_write(tmp_path, ONE_TET.format(tags="1 1", etype=5, extra=" 1 2 3 4")))
    with pytest.raises(ValueError, match="physical tags"):
        M.read_gmsh(_write(tmp_path, ONE_TET.format(tags="2 1 2", etype=4, extra="")))
    with pytest.raises(ValueError, match="skip numbers"):
        M.read_gmsh(_write(tmp_path, ONE_TET.format(tags="1 2", etype=4, extra="")))
    with pytest.raises(ValueError, match="MSH 4.1 ASCII"):
        M.read_gmsh(_write(tmp_path, ONE_TET.replace("4.1 0 8", "2.2 0 8").format(tags="1 1", etype=4, extra="")))


TWO_VOLUMES = """$MeshFormat
4.1 0 8
$EndMeshFormat
$Entities
0 0 0 2
1 0 0 0 1 1 1 0 0
2 0 0 0 1 1 1 {tags2} 0
$EndEntities
$Nodes
1 5 1 5
3 1 0 5
1
2
3
4
5
0 0 0
1 0 0
0 1 0
0 0 1
1 1 1
$EndNodes
$Elements
2 2 1 2
3 1 4 1
1 1 2 3 4
3 2 4 1
2 2 3 4 5
$EndElements
"""


def test_untagged_volume_is_material_one(tmp_path):
    """ReadGMSH.f90:119-139: a volume without a physical tag is material 1; it may sit next to
    volumes tagged 1, but not next to volumes of another material."""
    m = M.read_gmsh(_write(tmp_path, TWO_VOLUMES.format(tags2="1 1")))
    assert m.NE == 2 and m.Nm == 1 and np.all(m.mat == 0)
    assert m.neighbors[0].tolist().count(1) == 1 and m.neighbors[1].tolist().count(0) == 1
    with pytest.raises(ValueError, match="not for all"):
        M.read_gmsh(_write(tmp_path, TWO_VOLUMES.format(tags2="1 2")))
