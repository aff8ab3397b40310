"""The FP64 oracle pinned against the reference's own golden data and known answers (CPU only)."""
import numpy as np
import pytest

import oracle as O
from helpers import golden, rel_l2, scatter_mms, scatter_moment, transport_mms
from lionbolt_b200 import mesh as M
from lionbolt_b200 import problems as P


@pytest.mark.parametrize("L,fname", [(11, "ordinates_L11.txt"), (7, "ordinates_L7.txt")])
def test_ordinates_match_reference_log(L, fname):
    """SNPrep.f90:39-76 ordering and values == the tables printed in the reference's lb.out files."""
    k, w = O.sn_quadrature(L + 1, 2 * (L + 1))
    g = golden(fname)
    assert k.shape == g.shape
    assert np.abs(k - g).max() < 1e-15 + 5e-17 * 4
    assert abs(w.sum() - 4 * np.pi) < 1e-13


def test_slab_gauss_legendre_matches_reference_log():
    x, w = O.gauss_legendre(16)
    assert np.abs(x - golden("mu_slab_L15.txt")).max() < 1e-15
    assert abs(w.sum() - 2.0) < 1e-14


def test_yy_normalisation():
    """YY(i',i,l) = w(i')(2l+1)P_l(k.k')/(4pi): the l=0 kernel integrates to one over directions."""
    k, w = O.sn_quadrature(4, 8)
    Y = O.yy(k, w, 3)
    assert np.allclose(Y[0].sum(axis=1), 1.0, atol=1e-14)
    # symmetry of the unweighted kernel
    U = Y[2] / w[None, :]
    assert np.allclose(U, U.T, atol=1e-14)


def test_moment_factorisation_equals_dense_kernel():
    """K = M Sigma D with real spherical harmonics reproduces the dense YYS kernel (addition theorem)."""
    k, w = O.sn_quadrature(6, 12)
    Ls = 5
    sig = 0.9 * 0.8 ** np.arange(Ls + 1)
    Yd = O.yy(k, w, Ls)
    YYS = np.tensordot(sig, Yd, axes=1)                  # [i][i']
    Ysh = np.stack([O.real_sh(Ls, d) for d in k])         # [NI, nm]
    lofj = np.concatenate([[l] * (2 * l + 1) for l in range(Ls + 1)])
    K = Ysh @ np.diag(sig[lofj]) @ (Ysh * w[:, None]).T
    assert np.abs(K - YYS).max() < 1e-13


def test_scatter_mms_known_answer():
    """ScatterMMS.f90: K exp(r.k) -> 2 pi (e^t - e^-t)/t at L = 15 on the [-1,1]^3 cube."""
    m = M.box_mesh(2, 2, 2, (-1, -1, -1), (1, 1, 1))
    o = O.Oracle(m)
    L = 15
    k, w = O.sn_quadrature(L + 1, 2 * (L + 1))
    assert o.set_angular(k, w, L) == 0
    s = np.array([[scatter_moment(l) for l in range(L + 1)]])
    o.set_xs([1.0], s)
    psi, exact = scatter_mms(m, k)
    out = o.scatter_apply(psi)
    assert rel_l2(out, exact) < 1e-6


def test_transport_mms_converges():
    """TransportMMS.f90: T^{-1} of the Gaussian MMS source converges to exp(-A r^2) under refinement."""
    errs = []
    for n in (8, 16):
        m = M.box_mesh(n, n, n, (-1, -1, -1), (1, 1, 1))
        o = O.Oracle(m)
        k, w = O.sn_quadrature(4, 8)
        assert o.set_angular(k, w, 3) == 0
        o.set_xs([1e-10], np.zeros((1, 4)))
        src, exact = transport_mms(m, k)
        errs.append(rel_l2(o.transport_inv(src), exact))
    # second-order DG convergence once the Gaussian (width ~0.3) is resolved
    assert errs[1] < 0.3 * errs[0]
    assert errs[1] < 0.1


def test_fea_closed_form_matches_quadrature():
    """The mass-eliminated IC/IFM/IIM of FiniteElementAnalysis.f90 have the closed forms used by the
    CUDA sweep: everything follows from s_f = A_f n_f / V."""
    m = M.box_mesh(3, 2, 2, (0, 0, 0), (1.5, 1.0, 2.0))
    o = O.Oracle(m)
    g = o.geometry()
    F = [[0, 1, 2], [0, 1, 3], [0, 2, 3], [1, 2, 3]]
    rng = np.random.default_rng(0)
    worst = 0.0
    for e in range(m.NE):
        s = g["area"][e][:, None] * g["n"][e] / g["vol"][e]
        assert abs(g["vol"][e] - g["detJ"][e] / 6) < 1e-14
        om = rng.normal(size=3)
        om /= np.linalg.norm(om)
        c = s @ om
        Tc = 0.3 * np.eye(4) + np.array([[5 / 3 * c[3 - kk]] * 4 for kk in range(4)])
        To = 0.3 * np.eye(4) - sum(om[d] * g["IC"][e][d] for d in range(3))
        for f in range(4):
            if om @ g["n"][e][f] < 0:
                continue
            To += (om @ g["n"][e][f]) * g["IFM"][e][f]
            for kp in F[f]:
                for kk in F[f]:
                    Tc[kk, kp] += c[f] * (2 if kk == kp else 1 / 3)
                Tc[3 - f, kp] -= c[f] * 4 / 3
        worst = max(worst, np.abs(Tc - To).max() / np.abs(To).max())
    assert worst < 1e-12


def test_sweep_order_literal_equals_counting():
    m = M.box_mesh(4, 3, 5, (0, 0, 0), (2, 1.5, 2.5))
    k, w = O.sn_quadrature(4, 8)
    a, b = O.Oracle(m), O.Oracle(m)
    assert a.set_angular(k, w, 3, literal=True) == 0
    assert b.set_angular(k, w, 3, literal=False) == 0
    A, B = a.schedule(), b.schedule()
    for key in ("sl", "isl", "SAoffset", "UFoffset", "upfaces", "ipsf", "nlevels"):
        assert np.array_equal(A[key], B[key]), key


def test_oracle_gmres_and_si_agree():
    prob = P.config0()
    m = M.box_mesh(5, 5, 5, (0, 0, 0), (10, 10, 10))
    o = O.Oracle(m)
    assert o.set_angular(prob.k, prob.w, prob.Ng - 1) == 0
    o.set_xs(prob.sigt[0], prob.sigs[0, 0])
    rng = np.random.default_rng(3)
    q = rng.uniform(0, 1, size=m.NENK * prob.NI)
    xg, ig = o.boltzmann_solve(q, "GMRES", m=20, rtol=1e-11)
    xs, is_ = o.boltzmann_solve(q, "SI", rtol=1e-11)
    assert ig["status"] == 0 and is_["status"] == 0
    assert rel_l2(xg, xs) < 1e-8
    # the GMRES answer satisfies (I - T^-1 K) psi = T^-1 q
    r = o.boltzmann_matvec(xg) - o.transport_inv(q)
    assert np.linalg.norm(r) < 1e-9 * np.linalg.norm(xg)


# ---- moment-space restatement (used for the 768k-tet fixture) -------------------------------------
@pytest.mark.parametrize("case", ["config0", "two_material_jittered"])
def test_streamed_sweep_is_the_literal_sweep(case):
    """The natural-order per-direction sweep of the moment-space path gives the literal
    encode / Sweep / decode result bit for bit, and D is the quadrature sum of Y_j w psi."""
    from helpers import jittered
    if case == "config0":
        m, (k, w), sigt = P.config0().mesh, O.sn_quadrature(4, 8), [0.2]
    else:
        m = jittered(P.config1_small(n=(4, 4, 8)).mesh, 0.05)
        (k, w), sigt = O.sn_quadrature(4, 8), [0.05, 0.4]
    o = O.Oracle(m)
    assert o.set_angular(k, w, 3) == 0
    o.set_xs(sigt, np.zeros((m.Nm, 4)))
    q = np.random.default_rng(3).uniform(size=m.NENK * k.shape[0])
    y, psi = o.moment_transport(3, q=q, want_psi=True)
    assert np.array_equal(psi, o.transport_inv(q))
    Ysh = np.stack([O.real_sh(3, d) for d in k])
    assert rel_l2(y, (Ysh * w[:, None]).T @ psi.reshape(k.shape[0], -1)) < 1e-14


def test_moment_solve_matches_angular_solve():
    """config0 (6,000 tets, 80 directions, P3, c = 0.9): the moment-space GMRES and the literal
    angular-space GMRES of BoltzmannOp%MatInv converge to the same angular flux (<= 1e-10)."""
    prob = P.config0()
    m = prob.mesh
    o = O.Oracle(m)
    assert o.set_angular(prob.k, prob.w, prob.Ls) == 0
    o.set_xs(prob.sigt[0], prob.sigs[0, 0])
    q = np.random.default_rng(4).uniform(size=m.NENK * prob.NI)
    ref, info = o.boltzmann_solve(q, "GMRES", m=20, rtol=1e-13, atol=0.0)
    assert info["status"] == 0
    phi, psi, inf2 = o.moment_solve(prob.Ls, prob.sigs[0, 0], q=q, m=20, rtol=1e-13, want_psi=True)
    assert inf2["status"] == 0
    assert rel_l2(psi, ref) < 1e-10
    assert rel_l2(np.sqrt(4 * np.pi) * phi[0], o.fluence(ref)) < 1e-10


def test_moment_multigroup_matches_angular_multigroup():
    """The moment-space group loop (downscatter sources from resident group moments, beam first-
    collision source from Y(Omega_b)) against the literal angular-space loop with tapes, on the
    768k-tet problem's physics (P5, 2 materials, 4 groups) on a 6 x 6 x 12-hex box: <= 1e-10."""
    prob = P.config1_small(n=(6, 6, 12), G=4, Ng=6, Nc=12)
    o = O.Oracle(prob.mesh)
    assert o.set_angular(prob.k, prob.w, prob.Ls) == 0
    flux_ref, dose_ref, _ = o.multigroup(prob, "GMRES", m=20, rtol=1e-13)
    r = o.mg_moment(prob, m=20, rtol=1e-13, rtol_snap=1e-6)
    assert rel_l2(r["dose"], dose_ref) < 1e-10
    for g in range(prob.G):
        assert rel_l2(r["flux"][g], flux_ref[g]) < 1e-10, g
    # the 1e-6 snapshots are 1e-6 solves of the same groups: close, not equal, and cheaper
    assert 0 < rel_l2(r["dose_snap"], r["dose"]) < 1e-4
    assert np.all(r["iters_snap"] < r["iters"])


def test_dgemv_scattering_path_matches_loop_path():
    """The per-node dgemv loop of ScatteringAlgebra.f90:39-48 through the bundled OpenBLAS equals
    the oracle's own per-node loop, on all nodes and on a node range (other nodes untouched)."""
    prob = P.config1_small(n=(2, 2, 4))
    o = O.Oracle(prob.mesh)
    assert o.set_angular_no_schedule(prob.k, prob.w, prob.Ls) == 0
    o.set_xs(prob.sigt[0], prob.sigs[0, 0])
    x = np.random.default_rng(8).normal(size=prob.mesh.NENK * prob.NI)
    ref = o.scatter_apply(x)
    assert rel_l2(o.scatter_apply_dgemv(x), ref) < 1e-14
    n = prob.mesh.NENK
    part = o.scatter_apply_dgemv(x, 40, 100).reshape(prob.NI, n)
    xr, rr = x.reshape(prob.NI, n), ref.reshape(prob.NI, n)
    assert rel_l2(part[:, 40:100], rr[:, 40:100]) < 1e-14
    assert np.array_equal(part[:, :40], xr[:, :40]) and np.array_equal(part[:, 100:], xr[:, 100:])


def test_moment_fgmres_with_diagonal_preconditioner():
    """SPARSKIT fgmres (iters.f:2511-2795) in moment space with a fixed per-moment right
    preconditioner z_j = d_j v_j (d_j = 1 / (1 - 0.6 c g^l)) reaches the GMRES answer, across
    restarts (m = 5), along another iteration path."""
    prob = P.config0()
    o = O.Oracle(prob.mesh)
    assert o.set_angular_streamed(prob.k, prob.w) == 0
    o.set_sigt(prob.sigt[0])
    q = np.random.default_rng(6).uniform(size=prob.mesh.NENK * prob.NI)
    lofj = np.concatenate([[l] * (2 * l + 1) for l in range(prob.Ls + 1)])
    d = 1.0 / (1.0 - 0.6 * 0.9 * 0.8 ** lofj)
    phi_g, _, ig = o.moment_solve(prob.Ls, prob.sigs[0, 0], q=q, m=5, rtol=1e-11)
    phi_f, _, inf = o.moment_solve(prob.Ls, prob.sigs[0, 0], q=q, m=5, rtol=1e-11, pdiag=d)
    assert ig["status"] == 0 and inf["status"] == 0
    assert rel_l2(phi_f, phi_g) < 1e-9
    assert inf["iters"] != ig["iters"]


@pytest.mark.parametrize("nmat", [1, 2])
def test_beam_ray_tracing_matches_closed_form(nmat):
    """RayTracing.f90 TraceVector (Moller-Trumbore against region faces; the single-material branch
    and the per-material branch), Beer's law and the FCSSource projection against the closed form of
    a normally incident beam through layers aligned with the mesh (4 x 4 x 8 hexes, 1 cm).  The beam
    plane lies 1 cm before the mesh, as the reference's inputs place their beam origins outside the
    mesh (TraceVector drops a lone intersection at t ~ 0, RayTracing.f90:327-335)."""
    from helpers import layered_beam_reference
    mat = None if nmat == 1 else (lambda c: ((c[:, 2] > 2.0) & (c[:, 2] < 4.0)).astype(np.int32))
    m = M.box_mesh(4, 4, 8, (0, 0, 0), (4.0, 4.0, 8.0), material=mat, Nm=nmat)
    sig = [0.3] if nmat == 1 else [0.3, 0.8]
    o = O.Oracle(m)
    unc = o.beam_uncollided([2.0, 2.0, -1.0], [0, 0, 1.0], [1.0, 0, 0], [0, 1.0, 0], 2.5, 3.0, sig)
    layers = [(0.0, 8.0, 0.3)] if nmat == 1 else [(0.0, 2.0, 0.3), (2.0, 4.0, 0.8), (4.0, 8.0, 0.3)]
    ref = layered_beam_reference(m, (2.0, 2.0), (2.5, 3.0), layers)
    assert np.count_nonzero(ref) > 0 and np.count_nonzero(ref) < ref.size
    assert np.abs(unc - ref).max() < 1e-12
