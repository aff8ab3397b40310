"""Batched dose solves (lb_batch_*): many independent problems with their own meshes, quadratures,
group counts and beams, solved together, must reproduce the single-problem solver and the FP64
oracle.  Tolerances: 1e-5 relative L2 against the oracle (the stated flux/dose target); against the
single-problem GPU solver the difference is only reduction order inside GMRES (1e-6)."""
import numpy as np
import pytest

import oracle as O
from helpers import rel_l2
from lionbolt_b200 import BatchSolver, MultigroupSolver
from lionbolt_b200 import problems as P

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _small_batch(count=5, seed=7):
    return P.batch_problems(count=count, seed=seed, hmin=3, hmax=6, groups=(1, 3), orders=(8, 12))


def test_batch_matches_single_problem_solver():
    probs = _small_batch()
    assert len({p.NI for p in probs}) > 1 and len({p.G for p in probs}) > 1   # mixed quadratures and groups
    bs = BatchSolver()
    ids = [bs.add_problem(p) for p in probs]
    it = bs.solve(m=20, rtol=1e-8)
    info = bs.info()
    assert info["problems"] == len(probs) and info["graph_launches"] > 0 and info["sweep_threads"] in (512, 1024)
    for pid, prob in zip(ids, probs):
        mg = MultigroupSolver().set_problem(prob)
        it1 = mg.solve("GMRES", m=20, rtol=1e-8)
        f1, d1 = mg.results()
        fb, db = bs.results(pid)
        assert np.all(it[pid, :prob.G] > 0) and np.all(it[pid, prob.G:] == 0)
        assert np.abs(it[pid, :prob.G] - it1).max() <= 1, (it[pid], it1)
        assert rel_l2(db, d1) < 1e-6, pid
        for g in range(prob.G):
            assert rel_l2(fb[g], f1[g]) < 1e-6, (pid, g)


def test_batch_matches_oracle():
    probs = _small_batch(count=3, seed=11)
    bs = BatchSolver()
    ids = [bs.add_problem(p) for p in probs]
    bs.solve(m=20, rtol=1e-8)
    for pid, prob in zip(ids, probs):
        o = O.Oracle(prob.mesh)
        assert o.set_angular(prob.k, prob.w, prob.Ls) == 0
        flux_ref, dose_ref, _ = o.multigroup(prob, "GMRES", m=20, rtol=1e-11)
        fb, db = bs.results(pid)
        assert rel_l2(db, dose_ref) < TOL, pid
        for g in range(prob.G):
            assert rel_l2(fb[g], flux_ref[g]) < TOL, (pid, g)


def test_batch_resolve_is_repeatable():
    probs = _small_batch(count=3, seed=5)
    bs = BatchSolver()
    for p in probs:
        bs.add_problem(p)
    it1 = bs.solve(m=10, rtol=1e-7)
    d1 = [bs.results(i)[1] for i in range(len(probs))]
    it2 = bs.solve(m=10, rtol=1e-7)
    d2 = [bs.results(i)[1] for i in range(len(probs))]
    assert np.array_equal(it1, it2)
    for a, b in zip(d1, d2):
        assert rel_l2(a, b) < 1e-12
