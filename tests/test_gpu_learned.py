"""GPU tests of the learned right preconditioner: inference, preconditioner and training kernels
against the NumPy reference (tests/mlp_ref.py), and FGMRES with the trained network against
plain GMRES, which checks its answer.

Tolerances: the network runs in BF16 with FP32 accumulation, so kernel-vs-reference comparisons
allow for accumulation order (relative L2 2e-3 on outputs and gradients).  The solver with the
network must reproduce the plain-GMRES flux and dose to 1e-5 relative L2."""
import numpy as np
import pytest

import mlp_ref as R
from helpers import rel_l2
from lionbolt_b200 import AngularClass, MultigroupSolver, TransportOp, XSType
from lionbolt_b200 import _lib
from lionbolt_b200 import problems as P

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _random_weights(seed, scale=0.25):
    return np.random.default_rng(seed).uniform(-scale, scale, size=R.NPARAM).astype(np.float32)


def _features(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(n, R.NIN))
    x[:, 16:] = rng.uniform(0.0, 1.0, size=(n, 3))
    return x.astype(np.float32)


def test_forward_kernel_matches_reference():
    op = TransportOp()
    assert op.lp_nparams() == R.NPARAM == 6480
    w = _random_weights(1)
    op.lp_set_weights(w)
    assert np.array_equal(op.lp_get_weights(), w)
    for n in (1, 17, 1000):            # a partial 16-row tile, several tiles
        x = _features(n, n)
        y = op.lp_forward(x)
        ref, _ = R.forward(w, x)
        assert rel_l2(y, ref) < 2e-3, n
        assert np.abs(y - ref).max() < 1e-2 * np.abs(ref).max()


def test_gradient_kernel_matches_reference():
    """Training kernel (forward + backward, BF16 forward, FP32 backward) vs the FP64 reference."""
    op = TransportOp()
    w = _random_weights(2)
    op.lp_set_weights(w)
    for n in (5, 700):
        x = _features(n, 10 + n)
        t = np.random.default_rng(n).normal(size=(n, R.NOUT)).astype(np.float32)
        wt = np.random.default_rng(n + 1).uniform(0.0, 3.0, size=n).astype(np.float32)
        loss, g = op.lp_loss_grad(x, t, wt)
        lref, gref = R.loss_grad(w, x, t, wt)
        assert abs(loss - lref) < 1e-4 * abs(lref), (loss, lref)
        assert rel_l2(g, gref) < 2e-3, n
        # every parameter block carries gradient
        for a, b in ((R.OFF_W1, R.OFF_B1), (R.OFF_W2, R.OFF_B2), (R.OFF_W3, R.OFF_B3), (R.OFF_B3, R.NPARAM)):
            assert np.abs(g[a:b]).max() > 0


def test_preconditioner_kernel_matches_reference():
    prob = P.config1_small(n=(4, 4, 8), G=2, Ng=4, Nc=8)
    m = prob.mesh
    sigt, sigs = prob.within_group(1)
    op = TransportOp().Build(m, AngularClass(k=prob.k, w=prob.w), XSType(sigt, sigs))
    w = _random_weights(3)
    op.lp_set_weights(w)
    nm = (prob.Ls + 1) ** 2
    v = np.random.default_rng(4).normal(size=nm * m.NENK)
    z = op.lp_apply(v)
    zref = R.apply(w, v, m, sigt, sigs[:, 0], nm)
    assert rel_l2(z - v, zref - v) < 2e-3
    # moments above l = 3 pass through unchanged
    assert np.array_equal(z[16 * m.NENK:], v[16 * m.NENK:])


def test_fgmres_without_network_is_plain_gmres():
    prob = P.config1_small(n=(4, 4, 8), G=2, Ng=4, Nc=8)
    a = MultigroupSolver().set_problem(prob)
    it_a = a.solve("GMRES", m=20, rtol=1e-6)
    fa, da = a.results()
    it_b = a.solve("FGMRES_ML", m=20, rtol=1e-6)
    fb, db = a.results()
    # same method; only the sweep launch shape (autotuner trials in the first solve) may differ
    assert np.abs(it_a - it_b).max() <= 1
    assert rel_l2(db, da) < 1e-7


def _train_problems(G, n):
    """Training problems: the config1 physics with other seeds (cross sections) and slab positions."""
    out = []
    for k, slab in enumerate([(1.0, 2.0), (2.5, 3.5), (3.5, 5.0)]):
        out.append(P.multigroup_box(n=n, size=(0.5 * n[0], 0.5 * n[1], 0.5 * n[2]), G=G, Ng=6, Nc=12,
                                    seed=1000 + k, slab=slab, name=f"train{k}"))
    return out


def test_learned_preconditioner_trains_and_matches_plain_gmres():
    G, n = 4, (6, 6, 12)
    mg = MultigroupSolver()
    mg.lp_init(seed=7)
    total = 0
    for p in _train_problems(G, n):
        mg.set_problem(p)
        total = mg.lp_generate(samples_per_group=2000, iters=8, seed=total + 1)
    assert total == 3 * G * 2000
    x, t, wt = mg.lp_samples()
    assert np.all(np.isfinite(x)) and np.all(np.isfinite(t)) and np.all(wt >= 0)
    nz = (x[:, :16] ** 2).sum(axis=1) > 0
    assert np.allclose((x[nz, :16] ** 2).mean(axis=1), 1.0, rtol=1e-4)
    # sigma_s0 / sigma_t of every sample is one of the training problems' within-group ratios
    ratios = np.concatenate([p.sigs[g, g, :, 0] / p.sigt[g] for p in _train_problems(G, n) for g in range(G)])
    assert np.min(np.abs(x[:, 18:19] - ratios[None, :].astype(np.float32)), axis=1).max() < 1e-6
    loss = mg.lp_train(steps=1500, batch=2048, lr=3e-3, seed=11)
    assert np.all(np.isfinite(loss))
    first, last = loss[:20].mean(), loss[-50:].mean()
    print(f"\ntraining loss {first:.4g} -> {last:.4g} over {loss.size} steps on {total} samples")
    assert last < 0.8 * first

    # held-out problem: the config1 seed and slab on the same grid
    test = P.multigroup_box(n=n, size=(0.5 * n[0], 0.5 * n[1], 0.5 * n[2]), G=G, Ng=6, Nc=12,
                            slab=(2.5 * n[2] / 20, 3.5 * n[2] / 20), name="held_out")
    mg.set_problem(test)
    ref = MultigroupSolver().set_problem(test)
    it_plain = ref.solve("GMRES", m=20, rtol=1e-8)
    f_plain, d_plain = ref.results()
    it_ml = mg.solve("FGMRES_ML", m=20, rtol=1e-8)
    f_ml, d_ml = mg.results()
    print(f"operator applications per group: GMRES {list(it_plain)}  FGMRES+network {list(it_ml)}")
    assert rel_l2(d_ml, d_plain) < TOL
    for g in range(G):
        assert rel_l2(f_ml[g], f_plain[g]) < TOL, g
    # the untrained network (initial weights, close to the identity) for comparison
    mg.lp_init(seed=7)
    it_init = mg.solve("FGMRES_ML", m=20, rtol=1e-8)
    f_init, d_init = mg.results()
    print(f"untrained network: {list(it_init)}")
    assert rel_l2(d_init, d_plain) < TOL


def test_learned_path_is_gated_per_group_and_never_slower_in_applications():
    """Per-group gating from a held-out calibration problem, with plain GMRES's count as the learned
    path's budget: on a third problem the learned solve takes no more operator applications than
    plain GMRES, and gives its dose."""
    G, n = 4, (6, 6, 12)
    mg = MultigroupSolver()
    mg.lp_init(seed=7)
    total = 0
    for p in _train_problems(G, n):
        mg.set_problem(p)
        total = mg.lp_generate(samples_per_group=2000, iters=8, seed=total + 1)
    mg.lp_train(steps=600, batch=2048, lr=3e-3, seed=11)
    val = P.multigroup_box(n=n, size=(0.5 * n[0], 0.5 * n[1], 0.5 * n[2]), G=G, Ng=6, Nc=12, seed=4242,
                           slab=(1.0, 1.5), name="validation")
    mg.set_problem(val)
    plain_v, learned_v = mg.lp_calibrate(m=20, rtol=1e-6)
    assert np.all(plain_v > 0) and np.all(learned_v > 0)
    enabled = (1.1 * learned_v < plain_v).astype(np.int32)
    print(f"\nvalidation: GMRES {list(plain_v)}  FGMRES+network {list(learned_v)}  enabled {list(enabled)}")
    test = P.multigroup_box(n=n, size=(0.5 * n[0], 0.5 * n[1], 0.5 * n[2]), G=G, Ng=6, Nc=12,
                            slab=(2.5 * n[2] / 20, 3.5 * n[2] / 20), name="held_out")
    ref = MultigroupSolver().set_problem(test)
    it_plain = ref.solve("GMRES", m=20, rtol=1e-6)
    _, d_plain = ref.results()
    mg.set_problem(test)
    mg.lp_set_groups(enabled, budget=plain_v)
    it_gated = mg.solve("FGMRES_ML", m=20, rtol=1e-6)
    _, d_gated = mg.results()
    print(f"held out: GMRES {list(it_plain)}  gated learned path {list(it_gated)}")
    assert rel_l2(d_gated, d_plain) < TOL
    # groups without the network run plain GMRES; enabled groups won on the validation problem
    for g in range(G):
        if not enabled[g]:
            # the same plain GMRES (one more application at most when an earlier group's learned
            # answer shifted this group's source in the last digits)
            assert it_gated[g] <= it_plain[g] + (1 if enabled[:g].any() else 0), g
    assert it_gated.sum() <= it_plain.sum() + int(np.sum(enabled * plain_v))
