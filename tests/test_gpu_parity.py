"""GPU parity: the CUDA path through the C ABI against the FP64 oracle on the same seeded inputs.

Tolerances: the sweep and the moment contractions run in FP32 (split-BF16 tensor-core products
reproduce FP32), the Krylov iteration in FP64.  Results must agree with the FP64 oracle to
1e-5 relative L2 (the target stated for scalar flux and dose)."""
import numpy as np
import pytest

import oracle as O
from helpers import golden_mesh, jittered, rel_l2, scatter_mms, scatter_moment, transport_mms
from lionbolt_b200 import AngularClass, BoltzmannOp, MultigroupSolver, ScatteringOp, TransportOp, XSType
from lionbolt_b200 import _lib
from lionbolt_b200 import mesh as M
from lionbolt_b200 import problems as P

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _pair(m, k, w, sigt, sigs, L=None):
    """(oracle, product TransportOp/ScatteringOp/BoltzmannOp builder) on the same inputs."""
    L = sigs.shape[1] - 1 if L is None else L
    o = O.Oracle(m)
    assert o.set_angular(k, w, L) == 0
    o.set_xs(sigt, sigs)
    ang = AngularClass(k=k, w=w)
    xs = XSType(sigt, sigs)
    return o, ang, xs


SWEEP_CASES = {
    "one_hex": lambda: (M.box_mesh(1, 1, 1), P.quadrature(2, 4), np.array([1.0]), np.zeros((1, 1))),
    "cube_2x2x2": lambda: (M.box_mesh(2, 2, 2, (0, 0, 0), (1, 1, 1)), P.quadrature(4, 8), np.array([0.7]),
                           np.zeros((1, 1))),
    "config0": lambda: (P.config0().mesh, P.quadrature(8, 10), np.array([0.2]), np.zeros((1, 1))),
    "two_material": lambda: (P.config1_small(n=(6, 6, 12)).mesh, P.quadrature(6, 12), np.array([0.05, 0.135]),
                             np.zeros((2, 1))),
    "jittered": lambda: (jittered(M.box_mesh(6, 5, 4, (0, 0, 0), (3.0, 2.5, 2.0)), 0.07), P.quadrature(4, 8),
                         np.array([1.3]), np.zeros((1, 1))),
    "thin_air": lambda: (M.box_mesh(4, 4, 4, (0, 0, 0), (2, 2, 2)), P.quadrature(4, 8), np.array([1e-6]),
                         np.zeros((1, 1))),
    # a void material (sigma_t = 0) next to an absorber: pure streaming through half of the elements
    "void_region": lambda: (P.config1_small(n=(6, 6, 12)).mesh, P.quadrature(6, 12), np.array([0.0, 0.9]),
                            np.zeros((2, 1))),
}


@pytest.mark.parametrize("case", sorted(SWEEP_CASES))
def test_transport_inverse_matches_oracle(case):
    m, (k, w), sigt, sigs = SWEEP_CASES[case]()
    o, ang, xs = _pair(m, k, w, sigt, sigs)
    T = TransportOp().Build(m, ang, xs)
    rng = np.random.default_rng(7)
    q = rng.uniform(0.0, 1.0, size=m.NENK * k.shape[0])
    ref = o.transport_inv(q)
    out = q.copy()
    T.MatInv(out)
    assert rel_l2(out, ref) < TOL
    # the GPU path is the one that ran
    assert T.timers()["sweep"][1] >= 1


@pytest.mark.parametrize("cfg", range(24))
def test_every_sweep_schedule_matches_oracle(cfg, monkeypatch):
    """Each launch candidate of the sweep autotuner (levels, prefetching levels, element flags,
    grouped directions, dataflow, cluster levels with and without element prefetch) reproduces the oracle's T^{-1} on a two-material mesh."""
    monkeypatch.setenv("LB_SWEEP_CONFIG", str(cfg))
    m, (k, w), sigt, sigs = SWEEP_CASES["two_material"]()
    o, ang, xs = _pair(m, k, w, sigt, sigs)
    T = TransportOp().Build(m, ang, xs)
    q = np.random.default_rng(cfg).uniform(0.0, 1.0, size=m.NENK * k.shape[0])
    ref = o.transport_inv(q)
    out = q.copy()
    T.MatInv(out)
    assert rel_l2(out, ref) < TOL


CLUSTER_CONFIGS = range(14, 24)   # launch candidates of the cluster schedule (plain, type tables, prefetch)


def _sweep_case(m, k, w, sigt, seed):
    o, ang, xs = _pair(m, k, w, sigt, np.zeros((sigt.size, 1)))
    T = TransportOp().Build(m, ang, xs)
    q = np.random.default_rng(seed).uniform(0.0, 1.0, size=m.NENK * k.shape[0])
    out = q.copy()
    T.MatInv(out)
    assert rel_l2(out, o.transport_inv(q)) < TOL
    return T


@pytest.mark.parametrize("cfg", CLUSTER_CONFIGS)
def test_cluster_schedule_wide_levels_and_cyclic_blocks(cfg, monkeypatch):
    """The cluster schedule (6-tet blocks swept as units) against the oracle on a two-material
    32^3-hex box whose block levels (over a thousand blocks) take several passes of a CTA, on a
    jittered mesh whose block graphs have cycles in some directions (blocks on a cycle are swept
    element by element there), and on the reference's unstructured het_cube mesh (blocks grown from
    face neighbours, listed in a member table)."""
    monkeypatch.setenv("LB_SWEEP_CONFIG", str(cfg))
    k, w = P.quadrature(2, 4)
    two = M.box_mesh(32, 32, 32, (0, 0, 0), (4, 4, 4), material=lambda c: (c[:, 0] > 2.5).astype(np.int32), Nm=2)
    T = _sweep_case(two, k, w, np.array([0.3, 1.1]), cfg)
    assert T._h.mesh_types() == 12
    assert T._h.sweep_config()["schedule"].startswith("cluster levels")
    m, (k, w), sigt, sigs = SWEEP_CASES["jittered"]()
    T = _sweep_case(m, k, w, sigt, cfg + 20)
    assert T._h.sweep_config()["schedule"].startswith("cluster levels")
    het = golden_mesh("het_cube_spherical_beam")
    T = _sweep_case(het, *P.quadrature(2, 4), np.array([0.07, 0.19]), cfg + 40)
    assert T._h.sweep_config()["schedule"].startswith("cluster levels")


def test_transport_mms_matches_oracle():
    m = M.box_mesh(6, 6, 6, (-1, -1, -1), (1, 1, 1))
    k, w = P.quadrature(4, 8)
    o, ang, xs = _pair(m, k, w, np.array([1e-10]), np.zeros((1, 1)))
    src, exact = transport_mms(m, k)
    ref = o.transport_inv(src)
    out = src.copy()
    TransportOp().Build(m, ang, xs).MatInv(out)
    assert rel_l2(out, ref) < TOL
    assert abs(rel_l2(out, exact) - rel_l2(ref, exact)) < 1e-4


def test_transport_is_linear_and_zero_preserving():
    m = M.box_mesh(5, 5, 5, (0, 0, 0), (2, 2, 2))
    k, w = P.quadrature(4, 8)
    T = TransportOp().Build(m, AngularClass(k=k, w=w), XSType([0.4], np.zeros((1, 1))))
    z = np.zeros(m.NENK * k.shape[0])
    T.MatInv(z)
    assert not np.any(z)
    rng = np.random.default_rng(11)
    a, b = rng.uniform(size=z.size), rng.uniform(size=z.size)
    ta, tb, tab = a.copy(), b.copy(), (2 * a - 3 * b)
    T.MatInv(ta)
    T.MatInv(tb)
    T.MatInv(tab)
    assert rel_l2(tab, 2 * ta - 3 * tb) < 1e-5


@pytest.mark.parametrize("nmat", [1, 2])
def test_scattering_matches_oracle(nmat):
    """Nm = 1 follows the reference's dgemm path, Nm > 1 its per-node dgemv loop."""
    if nmat == 1:
        m = M.box_mesh(3, 3, 3, (0, 0, 0), (1, 1, 1))
        sigt, sigs = np.array([0.5]), np.array([[0.45 * 0.8 ** l for l in range(6)]])
    else:
        m = P.config1_small(n=(3, 3, 6)).mesh
        sigt = np.array([0.3, 0.81])
        sigs = np.array([[0.27 * 0.7 ** l for l in range(6)], [0.6 * 0.9 ** l for l in range(6)]])
    k, w = P.quadrature(6, 12)
    o, ang, xs = _pair(m, k, w, sigt, sigs, L=5)
    rng = np.random.default_rng(5)
    x = rng.normal(size=m.NENK * k.shape[0])
    ref = o.scatter_apply(x)
    out = x.copy()
    ScatteringOp().Build(m, ang, xs).MatVec(out)
    assert rel_l2(out, ref) < TOL


@pytest.mark.parametrize("nmat", [1, 2])
def test_device_contractions_compose_to_scattering(nmat):
    """lb_d2m_device then lb_m2d_device on caller-owned device arrays (asynchronous on the handle's
    stream; lb_synchronize reports their status) give K psi of the oracle."""
    torch = pytest.importorskip("torch")
    import ctypes
    if nmat == 1:
        m = M.box_mesh(3, 3, 3, (0, 0, 0), (1, 1, 1))
        sigt, sigs = np.array([0.5]), np.array([[0.45 * 0.8 ** l for l in range(6)]])
    else:
        m = P.config1_small(n=(3, 3, 6)).mesh
        sigt = np.array([0.3, 0.81])
        sigs = np.array([[0.27 * 0.7 ** l for l in range(6)], [0.6 * 0.9 ** l for l in range(6)]])
    k, w = P.quadrature(6, 12)
    o, ang, xs = _pair(m, k, w, sigt, sigs, L=5)
    x = np.random.default_rng(15).normal(size=m.NENK * k.shape[0]).astype(np.float32).astype(np.float64)
    ref = o.scatter_apply(x)
    K = ScatteringOp().Build(m, ang, xs)
    lib, h = K._h.lib, K._h.h
    psi = torch.from_numpy(x.astype(np.float32)).to("cuda:0")
    phi = torch.zeros(36 * m.NENK, dtype=torch.float64, device="cuda:0")
    out = torch.zeros_like(psi)
    torch.cuda.synchronize()
    assert lib.lb_d2m_device(h, ctypes.c_void_p(psi.data_ptr()), ctypes.c_void_p(phi.data_ptr())) == 0
    assert lib.lb_m2d_device(h, ctypes.c_void_p(phi.data_ptr()), ctypes.c_void_p(out.data_ptr())) == 0
    assert lib.lb_synchronize(h) == 0
    assert rel_l2(out.cpu().numpy(), ref) < TOL
    assert K.timers()["m2d"][1] >= 1 and K.timers()["d2m"][1] >= 1


def test_scatter_mms_known_answer_on_gpu():
    m = M.box_mesh(2, 2, 2, (-1, -1, -1), (1, 1, 1))
    L = 15
    k, w = P.quadrature(L + 1, 2 * (L + 1))
    s = np.array([[scatter_moment(l) for l in range(L + 1)]])
    K = ScatteringOp().Build(m, AngularClass(k=k, w=w), XSType([1.0], s))
    psi, exact = scatter_mms(m, k)
    out = psi.copy()
    K.MatVec(out)
    assert rel_l2(out, exact) < 2e-5


@pytest.mark.parametrize("solver", ["GMRES", "SI"])
def test_boltzmann_solve_matches_oracle(solver):
    prob = P.config0()
    m = prob.mesh
    o, ang, xs = _pair(m, prob.k, prob.w, prob.sigt[0], prob.sigs[0, 0])
    rng = np.random.default_rng(2)
    q = rng.uniform(0, 1, size=m.NENK * prob.NI)
    ref, info = o.boltzmann_solve(q, "GMRES", m=20, rtol=1e-11)
    assert info["status"] == 0
    L = BoltzmannOp(m=20, rtol=1e-8, atol=0.0).Build(m, ang, xs)
    out = q.copy()
    L.MatInv(out, solver=solver)
    assert L.iters > 1
    assert rel_l2(out, ref) < TOL
    fl, flr = o.fluence(out), o.fluence(ref)
    assert rel_l2(fl, flr) < TOL


def test_boltzmann_matvec_matches_oracle():
    m = M.box_mesh(3, 3, 3, (0, 0, 0), (3, 3, 3))
    k, w = P.quadrature(4, 8)
    sigt, sigs = np.array([0.6]), np.array([[0.5, 0.3, 0.1, 0.02]])
    o, ang, xs = _pair(m, k, w, sigt, sigs)
    x = np.random.default_rng(9).normal(size=m.NENK * k.shape[0])
    ref = o.boltzmann_matvec(x)
    out = x.copy()
    BoltzmannOp().Build(m, ang, xs).MatVec(out)
    assert rel_l2(out, ref) < TOL


def test_multigroup_flux_and_dose_match_oracle():
    prob = P.config1_small(n=(6, 6, 12), G=4, Ng=6, Nc=12)
    o = O.Oracle(prob.mesh)
    assert o.set_angular(prob.k, prob.w, prob.Ls) == 0
    flux_ref, dose_ref, it_ref = o.multigroup(prob, "GMRES", m=20, rtol=1e-11)
    mg = MultigroupSolver().set_problem(prob)
    it = mg.solve("GMRES", m=20, rtol=1e-8)
    flux, dose = mg.results()
    assert np.all(it > 0)
    assert rel_l2(dose, dose_ref) < TOL
    for g in range(prob.G):
        assert rel_l2(flux[g], flux_ref[g]) < TOL, g


def test_gmres_iteration_limit_reports_noconv():
    prob = P.config0()
    L = BoltzmannOp(m=5, rtol=1e-14, atol=0.0, maxit=3).Build(prob.mesh, AngularClass(k=prob.k, w=prob.w),
                                                              XSType(prob.sigt[0], prob.sigs[0, 0]))
    q = np.ones(prob.mesh.NENK * prob.NI)
    with pytest.raises(_lib.LionboltError) as ei:
        L.MatInv(q)
    assert ei.value.status == _lib.LB_ERR_NOCONV


@pytest.mark.parametrize("m", [5, 20])
def test_fgmres_pinned_to_sparskit_fgmres(m):
    """The device FGMRES(m) with a fixed per-moment diagonal right preconditioner (z_j = d_j v_j,
    d_j = 1 / (1 - 0.6 c g^l)) against the oracle's SPARSKIT fgmres (iters.f:2511-2795) in moment space
    with the same preconditioner, right-hand side D T^-1 q and initial guess: the same operator
    count to +-1, across restarts (m = 5), and the same angular flux to 1e-5."""
    prob = P.config0()
    mesh = prob.mesh
    o, ang, xs = _pair(mesh, prob.k, prob.w, prob.sigt[0], prob.sigs[0, 0])
    q = np.random.default_rng(12).uniform(0, 1, size=mesh.NENK * prob.NI)
    lofj = np.concatenate([[l] * (2 * l + 1) for l in range(prob.Ls + 1)])
    d = 1.0 / (1.0 - 0.6 * 0.9 * 0.8 ** lofj)
    _, psi_ref, info = o.moment_solve(prob.Ls, prob.sigs[0, 0], q=q, m=m, rtol=1e-6, pdiag=d, want_psi=True)
    assert info["status"] == 0
    L = BoltzmannOp(m=m, rtol=1e-6, atol=0.0).Build(mesh, ang, xs)
    L.set_right_precond_diag(d)
    out = q.copy()
    L.MatInv(out, solver="FGMRES")
    assert abs(L.iters - info["iters"]) <= 1, (L.iters, info["iters"])
    assert rel_l2(out, psi_ref) < TOL
    # the preconditioner is in effect: plain GMRES takes another number of operator applications
    _, _, plain = o.moment_solve(prob.Ls, prob.sigs[0, 0], q=q, m=m, rtol=1e-6)
    assert plain["iters"] != info["iters"]


def test_gmres_stagnation_below_the_fp32_floor_is_reported():
    """A tolerance below what the FP32 sweep resolves leaves the true residual at a floor: the solve
    stops after five restarts without progress with LB_ERR_NOCONV (this case used to cycle through
    about 200,000 operator applications before its residual dipped under 1e-8 by chance)."""
    import time
    prob = P.config1_small(n=(4, 4, 8), G=2, Ng=4, Nc=8)
    mg = MultigroupSolver().set_problem(prob)
    t0 = time.perf_counter()
    with pytest.raises(_lib.LionboltError) as ei:
        mg.solve("GMRES", m=20, rtol=1e-8)
    assert ei.value.status == _lib.LB_ERR_NOCONV and "stagnated" in str(ei.value)
    assert time.perf_counter() - t0 < 20
