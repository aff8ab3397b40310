"""The NumPy reference of the learned preconditioner, checked on its own (CPU only): backward pass
against central finite differences, BF16 rounding, and the mean-chord feature."""
import numpy as np

import mlp_ref as R
from lionbolt_b200 import mesh as M


def _weights(seed, scale=0.3):
    rng = np.random.default_rng(seed)
    return rng.uniform(-scale, scale, size=R.NPARAM)


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(1)
    w = _weights(0)
    x = rng.normal(size=(12, R.NIN))
    t = rng.normal(size=(12, R.NOUT))
    wt = rng.uniform(0.1, 2.0, size=12)
    _, g = R.loss_grad(w, x, t, wt, round=False)
    idx = rng.choice(R.NPARAM, size=120, replace=False)
    eps = 1e-6
    for p in idx:
        wp, wm = w.copy(), w.copy()
        wp[p] += eps
        wm[p] -= eps
        fd = (R.loss_grad(wp, x, t, wt, round=False)[0] - R.loss_grad(wm, x, t, wt, round=False)[0]) / (2 * eps)
        assert abs(fd - g[p]) <= 1e-6 * max(1.0, abs(g[p])), p


def test_bf16_rounding_is_nearest_even():
    vals = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -7, 1.0 + 3 * 2 ** -8, -2.5, 3.14159265])
    r = R.bf16(vals)
    assert r[0] == 1.0
    assert r[1] == 1.0                       # tie -> even mantissa
    assert r[2] == 1.0 + 2 ** -7
    assert r[3] == 1.0 + 2 ** -6             # tie -> even mantissa (rounds up)
    assert r[4] == -2.5
    assert abs(r[5] - 3.140625) < 1e-12


def test_mean_chord_of_a_unit_cube_split():
    m = M.box_mesh(1, 1, 1)
    ell = R.mean_chord(m)
    p = m.rg[m.node]
    vol = np.abs(np.einsum("ij,ij->i", np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), p[:, 3] - p[:, 0])) / 6
    assert np.allclose(vol.sum(), 1.0)
    assert np.all(ell > 0) and np.all(ell < 1.0)


def test_feature_scale_normalises_moments():
    m = M.box_mesh(2, 2, 2)
    nm = 16
    v = np.random.default_rng(3).normal(size=nm * m.NENK)
    x, s = R.features(v, m, [0.5], [0.3], nm)
    assert np.allclose((x[:, :16] ** 2).mean(axis=1), 1.0)
    assert np.allclose(x[:, 18], 0.6)
