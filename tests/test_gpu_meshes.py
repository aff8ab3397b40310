"""The CUDA path on the reference's own unstructured gmsh meshes (general element shapes: 64-byte
element records, element-level schedules), against the FP64 oracle on the same inputs.

  simple_cube.msh               validation/operators/simple_cube.msh, 12,741 tets
  het_cube_spherical_beam.msh   examples/water_tank_with_aluminum/het_cube_spherical_beam.msh,
                                78,771 tets, 2 materials

Both are read from tests/golden fixtures (tests/golden/make_mesh_fixtures.py).  Tolerance: 1e-5
relative L2 (FP32 sweep against FP64)."""
import numpy as np
import pytest

import oracle as O
from helpers import golden_mesh, rel_l2, transport_mms
from lionbolt_b200 import AngularClass, BoltzmannOp, TransportOp, XSType
from lionbolt_b200 import problems as P

pytestmark = pytest.mark.gpu

TOL = 1e-5


def test_transport_mms_on_the_reference_simple_cube():
    """validation/operators/TransportMMS.f90:44-89 as the reference runs it: simple_cube.msh scaled
    by 2 (mesh%Scale), AngularClass(15) = 512 directions, sigma = 1e-10, Gaussian MMS with A = 10."""
    m = golden_mesh("simple_cube")
    m.rg = m.rg * 2.0
    assert (m.NE, m.NN) == (12741, 2786)
    k, w = P.quadrature(16, 32)
    o = O.Oracle(m)
    assert o.set_angular(k, w, 0, literal=False) == 0
    o.set_xs([1e-10], np.zeros((1, 1)))
    src, exact = transport_mms(m, k)
    ref = o.transport_inv(src)
    T = TransportOp().Build(m, AngularClass(k=k, w=w), XSType([1e-10], np.zeros((1, 1))))
    assert T._h.mesh_types() == 0          # general shapes: 64-byte element records
    out = src.copy()
    T.MatInv(out)
    assert rel_l2(out, ref) < TOL
    # the discretisation error against the closed form is the oracle's (a few percent on this mesh)
    e_gpu, e_ref = rel_l2(out, exact), rel_l2(ref, exact)
    assert e_ref < 0.2
    assert abs(e_gpu - e_ref) < 1e-4 * e_ref + 1e-6


@pytest.fixture(scope="module")
def het_cube():
    m = golden_mesh("het_cube_spherical_beam")
    assert (m.NE, m.Nm) == (78771, 2)
    return m


def test_transport_inverse_on_the_reference_het_cube(het_cube):
    m = het_cube
    k, w = P.quadrature(8, 16)
    sigt = np.array([0.07, 0.19])
    o = O.Oracle(m)
    assert o.set_angular(k, w, 0, literal=False) == 0
    o.set_xs(sigt, np.zeros((2, 1)))
    q = np.random.default_rng(21).uniform(size=m.NENK * k.shape[0])
    ref = o.transport_inv(q)
    out = q.copy()
    TransportOp().Build(m, AngularClass(k=k, w=w), XSType(sigt, np.zeros((2, 1)))).MatInv(out)
    assert rel_l2(out, ref) < TOL


def test_boltzmann_solve_on_the_reference_het_cube(het_cube):
    """A within-group solve (c = 0.9, P3 Henyey-Greenstein g = 0.8) on the two-material mesh against
    the moment-space FP64 oracle solved to 1e-11."""
    m = het_cube
    k, w = P.quadrature(6, 12)
    sigt = np.array([0.07, 0.19])
    sigs = np.array([[0.9 * s * 0.8 ** l for l in range(4)] for s in sigt])
    o = O.Oracle(m)
    assert o.set_angular_streamed(k, w) == 0
    o.set_sigt(sigt)
    q = np.random.default_rng(22).uniform(size=m.NENK * k.shape[0])
    _, psi_ref, info = o.moment_solve(3, sigs, q=q, m=20, rtol=1e-11, want_psi=True)
    assert info["status"] == 0
    L = BoltzmannOp(m=20, rtol=1e-8, atol=0.0).Build(m, AngularClass(k=k, w=w), XSType(sigt, sigs))
    out = q.copy()
    L.MatInv(out)
    assert rel_l2(out, psi_ref) < TOL
