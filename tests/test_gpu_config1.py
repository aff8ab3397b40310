"""Parity at the benchmarked problem: the 768,000-tet, 288-direction, 20-group P5 dose solve on the
GPU (FP32 sweep, split-BF16 tensor-core moments, FP64 Krylov, GMRES(20) to a 1e-6 moment residual)
against the FP64 oracle's converged (1e-10) solution of the same problem.

The oracle's full solution is 1 GB and takes over an hour on CPU cores, so it is stored as a
fixture (tests/golden/config1_oracle.npz, made by tests/golden/make_config1_fixture.py): the dose and
every group's scalar fluence at 4096 seeded DG nodes, their sums over every hex layer along z (every
node enters one), the full-vector norms, and a SHA-256 of the level-set element order of all 288
directions.  Tolerance: 1e-5 relative L2 for flux and dose; element orderings bit-exact.

A second test runs the same physics (288 directions, 20 groups, P5, c = 0.9, g up to 0.95) on an
8 x 8 x 16-hex box against the moment-space FP64 oracle run in the test, on every node."""
import hashlib
import os

import numpy as np
import pytest

import oracle as O
from helpers import GOLDEN, rel_l2
from lionbolt_b200 import MultigroupSolver
from lionbolt_b200 import problems as P

pytestmark = pytest.mark.gpu

TOL = 1e-5
FIXTURE = os.path.join(GOLDEN, "config1_oracle.npz")


def layer_sums(v, shape):
    nx, ny, nz = shape
    return v.reshape(nz, -1).sum(axis=1)


@pytest.mark.skipif(not os.path.exists(FIXTURE), reason="config1 oracle fixture not generated")
def test_config1_flux_and_dose_match_fp64_oracle():
    d = np.load(FIXTURE)
    prob = P.config1()
    mg = MultigroupSolver().set_problem(prob)
    # element orderings: the level sets of all 288 directions, bit for bit
    sl, _, nl, _ = mg.schedule()
    assert np.array_equal(nl, d["nlevels"])
    assert hashlib.sha256(np.ascontiguousarray(sl, dtype="<i4").tobytes()).hexdigest() == str(d["sl_sha256"])
    del sl
    it = mg.solve("GMRES", m=20, rtol=1e-6)
    assert np.all(it > 0)
    flux, dose = mg.results()
    nodes = d["nodes"]
    shape = prob.mesh.shape
    errs = {"dose": rel_l2(dose[nodes], d["dose"]),
            "dose_layers": rel_l2(layer_sums(dose, shape), d["dose_layers"])}
    for g in range(prob.G):
        errs[f"flux{g}"] = rel_l2(flux[g, nodes], d["flux"][g])
        errs[f"flux{g}_layers"] = rel_l2(layer_sums(flux[g], shape), d["flux_layers"][g])
        assert abs(np.linalg.norm(flux[g]) / d["flux_norm"][g] - 1) < TOL, g
    assert abs(np.linalg.norm(dose) / float(d["dose_norm"]) - 1) < TOL
    print("rel. L2 vs the FP64 oracle:", {k: f"{v:.2e}" for k, v in errs.items()})
    bad = {k: v for k, v in errs.items() if not v < TOL}
    assert not bad, bad


def test_config1_physics_on_a_small_box_matches_fp64_oracle():
    prob = P.multigroup_box(n=(8, 8, 16), size=(4.0, 4.0, 8.0), slab=(1.0, 1.4), name="config1 physics 8x8x16")
    assert prob.NI == 288 and prob.G == 20 and prob.nm == 36
    o = O.Oracle(prob.mesh)
    assert o.set_angular_streamed(prob.k, prob.w) == 0
    ref = o.mg_moment(prob, m=20, rtol=1e-10)
    mg = MultigroupSolver().set_problem(prob)
    mg.solve("GMRES", m=20, rtol=1e-6)
    flux, dose = mg.results()
    assert rel_l2(dose, ref["dose"]) < TOL
    for g in range(prob.G):
        assert rel_l2(flux[g], ref["flux"][g]) < TOL, g
