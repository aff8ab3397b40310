"""The Arnoldi orthogonalisation of the device GMRES, restated in FP64 NumPy on the oracle's operator.

The device solver projects each new Krylov vector once, with coefficients c = G^{-1} V^T w where
G = V^T V is the basis' Gram matrix (kept from the dots of the projection pass), instead of projecting
twice (classical Gram-Schmidt with re-orthogonalisation).  This test restates both forms as GMRES(20)
on the angular operator x -> x - T^{-1} K x of the FP64 oracle and checks that they take the same
number of operator applications and reach the same true residual, at the 1e-6 target and at 1e-10
(the tolerance the learned preconditioner's training data uses), and that the device's bookkeeping with
unnormalised stored basis vectors (scale factors in the coefficients) gives the same iteration.  CPU only;
the oracle is the checker.
"""
import numpy as np
import pytest

import oracle as O
from lionbolt_b200 import problems as P


def _gmres(apply_a, b, m, rtol, gram, maxmv=200):
    x = np.zeros_like(b)
    nmv = 0
    bn = np.linalg.norm(b)
    while True:
        r = b - apply_a(x)
        nmv += 1
        beta = np.linalg.norm(r)
        if beta <= rtol * bn or nmv > maxmv:
            return nmv, beta / bn
        V = [r / beta]
        H = np.zeros((m + 1, m))
        G = np.eye(m + 1)
        g = np.zeros(m + 1)
        g[0] = beta
        for k in range(m):
            w = apply_a(V[k])
            nmv += 1
            Vm = np.array(V)
            h = Vm @ w
            if gram:
                c = np.linalg.solve(G[:k + 1, :k + 1], h)
                w2 = w - Vm.T @ c
                h2 = Vm @ w2
            else:   # classical Gram-Schmidt, second projection when the first cancelled over half of |w|^2
                w2 = w - Vm.T @ h
                h2 = Vm @ w2
                if w2 @ w2 < 0.5 * (w @ w):
                    w2 = w2 - Vm.T @ h2
                    h = h + h2
                c = h
            hk = np.linalg.norm(w2)
            H[:k + 1, k] = c
            H[k + 1, k] = hk
            if gram:
                G[:k + 1, k + 1] = G[k + 1, :k + 1] = h2 / hk
            V.append(w2 / hk)
            y = np.linalg.lstsq(H[:k + 2, :k + 1], g[:k + 2], rcond=None)[0]
            if np.linalg.norm(g[:k + 2] - H[:k + 2, :k + 1] @ y) <= rtol * bn or k == m - 1 or nmv > maxmv:
                x = x + np.array(V[:k + 1]).T @ y
                break


def _gmres_deferred(apply_a, b, m, rtol, maxmv=200):
    """The device's bookkeeping: the stored basis vectors W_i are not normalised (V_i = sc_i W_i), the
    scale factors enter the coefficients of the dot and axpy passes, the Hessenberg column and the Gram
    matrix, and the solution update; no pass divides a vector by its norm."""
    x = np.zeros_like(b)
    nmv = 0
    bn = np.linalg.norm(b)
    while True:
        r = b - apply_a(x)
        nmv += 1
        beta = np.linalg.norm(r)
        if beta <= rtol * bn or nmv > maxmv:
            return nmv, beta / bn
        W, sc = [r], [1.0 / beta]
        H = np.zeros((m + 1, m))
        G = np.eye(m + 1)
        g = np.zeros(m + 1)
        g[0] = beta
        for k in range(m):
            w = apply_a(W[k])                      # = A V_k / sc_k
            nmv += 1
            s1 = sc[k]
            Wm, scv = np.array(W), np.array(sc)
            h = (Wm @ w) * scv * s1                # V^T (A V_k)
            c = np.linalg.solve(G[:k + 1, :k + 1], h)
            w = w - Wm.T @ (c * scv / s1)
            h2 = (Wm @ w) * scv * s1
            hk = s1 * np.linalg.norm(w)
            H[:k + 1, k] = c
            H[k + 1, k] = hk
            G[:k + 1, k + 1] = G[k + 1, :k + 1] = h2 / hk
            W.append(w)
            sc.append(s1 / hk)
            y = np.linalg.lstsq(H[:k + 2, :k + 1], g[:k + 2], rcond=None)[0]
            if np.linalg.norm(g[:k + 2] - H[:k + 2, :k + 1] @ y) <= rtol * bn or k == m - 1 or nmv > maxmv:
                x = x + np.array(W[:k + 1]).T @ (y * np.array(sc[:k + 1]))
                break


@pytest.mark.parametrize("rtol", [1e-6, 1e-10])
def test_gram_corrected_projection_converges_like_reorthogonalised(rtol):
    prob = P.config1_small(n=(4, 4, 8), G=4, Ng=4, Nc=8)
    o = O.Oracle(prob.mesh)
    assert o.set_angular(prob.k, prob.w, prob.Ls) == 0
    o.set_xs(*prob.within_group(prob.G - 1))   # the most strongly scattering group
    apply_a = lambda x: x - o.transport_inv(o.scatter_apply(x))
    b = o.transport_inv(np.random.default_rng(3).uniform(0.0, 1.0, prob.mesh.NENK * prob.NI))
    n_re, r_re = _gmres(apply_a, b, 20, rtol, gram=False)
    n_gr, r_gr = _gmres(apply_a, b, 20, rtol, gram=True)
    n_df, r_df = _gmres_deferred(apply_a, b, 20, rtol)
    assert r_re <= rtol and r_gr <= rtol and r_df <= rtol
    assert n_gr == n_re and n_df == n_gr
    assert abs(r_gr - r_re) <= 1e-3 * r_re
    assert abs(r_df - r_gr) <= 1e-6 * r_gr     # the deferred normalisation changes only rounding
