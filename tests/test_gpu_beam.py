"""The first-collision data of a planar beam ray-traced on the GPU (lb_beam_uncollided: tet-to-tet walk
in FP64) against the oracle's literal restatement of the reference's ray tracing (TraceVector,
RayTracing.f90:205-379: Moller-Trumbore against every region-boundary face), Beer's law and the
FCSSource projection, and against the closed form for layered media.  Both sides are FP64, so the
tolerance is 1e-10 absolute on values <= 1 (rounding of different intersection arithmetic)."""
import numpy as np
import pytest

import oracle as O
from helpers import golden_mesh, layered_beam_reference, rel_l2
from lionbolt_b200 import AngularClass, MultigroupSolver, TransportOp
from lionbolt_b200 import mesh as M
from lionbolt_b200 import problems as P

pytestmark = pytest.mark.gpu

ATOL = 1e-10


def _frame(theta_deg, phi_deg=0.0):
    th, ph = np.deg2rad(theta_deg), np.deg2rad(phi_deg)
    axis = np.array([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)])
    e1 = np.cross([0.0, 1.0, 0.0], axis)
    e1 /= np.linalg.norm(e1)
    e2 = np.cross(axis, e1)
    return axis, e1, e2


def _op(m):
    k, w = P.quadrature(2, 4)
    return TransportOp().Build(m, AngularClass(k=k, w=w))


def test_layered_box_matches_closed_form_and_oracle():
    m = M.box_mesh(4, 4, 8, (0, 0, 0), (4.0, 4.0, 8.0),
                   material=lambda c: ((c[:, 2] > 2.0) & (c[:, 2] < 4.0)).astype(np.int32), Nm=2)
    args = ([2.0, 2.0, -1.0], [0, 0, 1.0], [1.0, 0, 0], [0, 1.0, 0], 2.5, 3.0, [0.3, 0.8])
    gpu = _op(m).beam_uncollided(*args)
    ref = layered_beam_reference(m, (2.0, 2.0), (2.5, 3.0), [(0.0, 2.0, 0.3), (2.0, 4.0, 0.8), (4.0, 8.0, 0.3)])
    assert np.abs(gpu - ref).max() < 1e-12
    assert np.abs(gpu - O.Oracle(m).beam_uncollided(*args)).max() < ATOL


@pytest.mark.parametrize("theta", [15.0, 37.0])
def test_oblique_beam_on_a_two_material_box_matches_oracle(theta):
    prob = P.config1_small(n=(6, 6, 12))
    m = prob.mesh
    axis, e1, e2 = _frame(theta, 20.0)
    # the beam plane beyond the mesh (40 cm from its centre along the axis; half its diagonal is 24.5 cm),
    # as the reference's inputs place their beam origins: TraceVector counts no path in a region whose
    # boundary the segment does not cross, so a plane through the mesh would leave such points unattenuated
    origin = np.array([10.0, 10.0, 20.0]) - 40.0 * axis
    args = (origin, axis, e1, e2, 9.0, 7.0, [0.11, 0.297])
    gpu = _op(m).beam_uncollided(*args)
    ref = O.Oracle(m).beam_uncollided(*args)
    assert 500 < np.count_nonzero(ref) < ref.size
    assert np.abs(gpu - ref).max() < ATOL


def test_reference_het_cube_mesh_matches_oracle():
    m = golden_mesh("het_cube_spherical_beam")                   # unit cube, 78,771 tets, 2 materials
    axis, e1, e2 = _frame(25.0, 40.0)
    origin = np.array([0.5, 0.5, 0.5]) - 1.5 * axis
    args = (origin, axis, e1, e2, 0.3, 0.25, [0.2, 0.54])
    gpu = _op(m).beam_uncollided(*args)
    ref = O.Oracle(m).beam_uncollided(*args)
    assert np.count_nonzero(ref) > 1000
    assert np.abs(gpu - ref).max() < ATOL


def test_single_material_branch_on_the_reference_simple_cube():
    m = golden_mesh("simple_cube")                               # [-0.5, 0.5]^3
    axis, e1, e2 = _frame(10.0, 0.0)
    args = (-1.0 * axis, axis, e1, e2, 0.6, 0.5, [0.7])
    gpu = _op(m).beam_uncollided(*args)
    ref = O.Oracle(m).beam_uncollided(*args)
    assert np.abs(gpu - ref).max() < ATOL


def test_ray_traced_source_drives_the_multigroup_solve():
    """lb_beam_uncollided leaves its result as the problem's uncollided flux: the dose solve with it
    equals the solve given the same values from the host."""
    prob = P.multigroup_box(n=(4, 4, 8), size=(4.0, 4.0, 8.0), G=3, Ng=4, Nc=8, slab=(2.0, 4.0), beam_deg=0.0)
    origin, axis, e1, e2 = [2.0, 2.0, -1.0], [0, 0, 1.0], [1.0, 0, 0], [0, 1.0, 0]
    mg = MultigroupSolver().set_problem(prob)
    unc = mg.beam_uncollided(origin, axis, e1, e2, 2.5, 2.5, prob.sigt[0])
    mg.solve("GMRES", m=20, rtol=1e-8)
    f1, d1 = mg.results()
    prob.unc = unc
    mg2 = MultigroupSolver().set_problem(prob)
    mg2.solve("GMRES", m=20, rtol=1e-8)
    f2, d2 = mg2.results()
    assert rel_l2(d1, d2) < 1e-12 and rel_l2(f1, f2) < 1e-12
