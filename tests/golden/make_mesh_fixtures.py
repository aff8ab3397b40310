"""Regenerates the mesh fixtures of the reference's two shipped unstructured meshes.

  mesh_simple_cube.npz              validation/operators/simple_cube.msh (12,741 tets; the mesh of
                                    the reference's TransportMMS driver)
  mesh_het_cube_spherical_beam.npz  examples/water_tank_with_aluminum/het_cube_spherical_beam.msh
                                    (78,771 tets, 2 materials)

Each holds the node coordinates (rg, float64), the connectivity (node, int32, gmsh order) and the
0-based materials (mat, uint8) exactly as lionbolt_b200.mesh.read_gmsh returns them; neighbours are
rebuilt by face matching when a test loads the fixture (tests/helpers.py golden_mesh), so tests that
run without the reference tree (the GPU box) sweep the same meshes.

Run from anywhere:  python tests/golden/make_mesh_fixtures.py <Lionbolt source root>
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from lionbolt_b200.mesh import read_gmsh  # noqa: E402

MESHES = {
    "simple_cube": "validation/operators/simple_cube.msh",
    "het_cube_spherical_beam": "examples/water_tank_with_aluminum/het_cube_spherical_beam.msh",
}


def main():
    if len(sys.argv) < 2:
        sys.exit("usage: make_mesh_fixtures.py <Lionbolt source root>")
    root = sys.argv[1]
    for name, rel in MESHES.items():
        m = read_gmsh(os.path.join(root, rel))
        out = os.path.join(HERE, f"mesh_{name}.npz")
        np.savez_compressed(out, rg=m.rg, node=m.node.astype(np.int32), mat=m.mat.astype(np.uint8))
        print(f"{out}: {m.NE} tets, {m.NN} nodes, {m.Nm} materials, {os.path.getsize(out)} bytes")


if __name__ == "__main__":
    main()
