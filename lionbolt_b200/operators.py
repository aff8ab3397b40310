"""Python mirror of the reference's operator API (src/LionboltAPI.f90 re-exports).

    TransportOp   T   Build(mesh, angular, XS) / MatInv(s)            TransportOperator.f90
    ScatteringOp  K   Build(mesh, angular, XS) / MatVec(x)            ScatteringOperator.f90
    BoltzmannOp   L   Build(mesh, angular, XS) / MatVec(x) / MatInv(s) BoltzmannOperator.f90
    SpaceAngleVector(mesh, angular) with .v and .Fluence(w)            LinearOperatorClass.f90

Vectors are FP64 numpy arrays in the reference layout v[i*NENK + 4e + k]; operations are in
place ("enters as source, leaves as solution", TransportAlgebra.f90:44).  Every call goes through
the C ABI to the CUDA library; errors raise LionboltError (the reference calls stophere).
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import as_f64, as_i32, dptr, iptr


class AngularClass:
    """SN quadrature, SNPrep.f90:39-86: AngularClass(L) gives Ng = L+1, Nc = 2 Ng; (Ng, Nc) may be
    given explicitly for direction counts the reference's tied construction cannot make."""

    def __init__(self, L=None, solver="GMRES", Ng=None, Nc=None, k=None, w=None):
        if k is not None:
            self.k, self.w = as_f64(k), as_f64(w)
            self.L = L if L is not None else -1
        else:
            if Ng is None:
                Ng = L + 1
            if Nc is None:
                Nc = 2 * Ng
            self.k, self.w = _lib.sn_quadrature(Ng, Nc)
            self.L = Ng - 1 if L is None else L
        self.solver = solver

    @property
    def NI(self):
        return int(self.k.shape[0])


class XSType:
    """Within-group cross sections: t[Nm] (XS%t) and s[Nm, L+1] (XS%s(0:L, m))."""

    def __init__(self, t, s):
        self.t = as_f64(np.atleast_1d(t))
        self.s = as_f64(np.atleast_2d(s))

    @property
    def L(self):
        return self.s.shape[1] - 1


class SpaceAngleVector:
    def __init__(self, mesh, angular, v=None):
        self.NENK = mesh.NENK
        self.NI = angular.NI
        self.v = np.zeros(self.NENK * self.NI) if v is None else as_f64(v).copy()

    def Fluence(self, w):
        """fl = sum_i w_i v_i (LinearOperatorClass.f90:154-174)."""
        return (np.asarray(w)[:, None] * self.v.reshape(self.NI, self.NENK)).sum(axis=0)


class _Op:
    name = "Operator"

    def __init__(self, device=0):
        self._h = _lib.Handle(device)
        self.mesh = None
        self.angular = None
        self.XS = None

    def Build(self, mesh, angular=None, XS=None):
        """Generic Build => Space / SpaceAngle / Physics, as the reference's generic interface."""
        h = self._h
        if mesh is not None and mesh is not self.mesh:
            h.call("lb_set_mesh", mesh.NE, mesh.NN, dptr(as_f64(mesh.rg)), iptr(as_i32(mesh.node)),
                   iptr(as_i32(mesh.neighbors)), iptr(as_i32(mesh.mat)), int(mesh.Nm))
            self.mesh = mesh
            self.angular = None
        if angular is not None and angular is not self.angular:
            h.call("lb_set_quadrature", angular.NI, dptr(angular.k), dptr(angular.w))
            self.angular = angular
        if XS is not None:
            self.set_xs(XS)
        return self

    def set_xs(self, XS):
        t = as_f64(XS.t)
        s = as_f64(XS.s)
        self._h.call("lb_set_xs", int(s.shape[1] - 1), dptr(t), dptr(s))
        self.XS = XS

    def _vec(self, s):
        v = s.v if isinstance(s, SpaceAngleVector) else s
        if not (isinstance(v, np.ndarray) and v.dtype == np.float64 and v.flags.c_contiguous):
            raise TypeError("vectors must be contiguous float64 numpy arrays")
        if v.size != self.mesh.NENK * self.angular.NI:
            raise ValueError("vector size does not match NENK*NI")
        return v

    def schedule(self):
        """(sl [NI, NE], upmask [NI, NE], nlevels [NI], level_start [NI, NE+1])"""
        NE, NI = self.mesh.NE, self.angular.NI
        sl = np.zeros((NI, NE), dtype=np.int32)
        up = np.zeros((NI, NE), dtype=np.uint8)
        nl = np.zeros(NI, dtype=np.int32)
        ls = np.zeros((NI, NE + 1), dtype=np.int32)
        self._h.call("lb_get_schedule", iptr(sl), up.ctypes.data_as(_lib._c_ubyte_p), iptr(nl), iptr(ls))
        return sl, up, nl, ls

    def timers(self):
        return self._h.timers()

    def beam_uncollided(self, origin, axis, e1, e2, width1, width2, attn):
        """Uncollided fluence [NENK] of a planar rectangular beam at the DG nodes, ray-traced on the device
        (RayTracing.f90, FluenceQuadrature.f90, FCSSource.f90); it also becomes the uncollided flux of
        the handle's multigroup problem."""
        args = [as_f64(np.asarray(v, dtype=np.float64).ravel()) for v in (origin, axis, e1, e2)]
        at = as_f64(np.atleast_1d(np.asarray(attn, dtype=np.float64)))
        unc = np.zeros(self.mesh.NENK)
        self._h.call("lb_beam_uncollided", *[dptr(a) for a in args], float(width1), float(width2), dptr(at), dptr(unc))
        return unc

    # ---- learned right preconditioner (per-cell MLP, used by solver="FGMRES_ML") ----------------
    NIN, NOUT = 19, 16

    def lp_nparams(self):
        return int(self._h.lib.lb_lp_nparams())

    def lp_init(self, seed=0):
        self._h.call("lb_lp_init", int(seed))
        return self

    def lp_set_weights(self, w):
        w = _lib.as_f32(w).ravel()
        if w.size != self.lp_nparams():
            raise ValueError(f"expected {self.lp_nparams()} parameters, got {w.size}")
        self._h.call("lb_lp_set_weights", _lib.fptr(w))
        return self

    def lp_get_weights(self):
        w = np.zeros(self.lp_nparams(), dtype=np.float32)
        self._h.call("lb_lp_get_weights", _lib.fptr(w))
        return w

    def lp_enable(self, on=True):
        self._h.call("lb_lp_enable", int(bool(on)))
        return self

    def lp_forward(self, x):
        """Network outputs [n, 16] for features x [n, 19] (tensor-core inference kernel)."""
        x = _lib.as_f32(x).reshape(-1, self.NIN)
        y = np.zeros((x.shape[0], self.NOUT), dtype=np.float32)
        self._h.call("lb_lp_forward", int(x.shape[0]), _lib.fptr(x), _lib.fptr(y))
        return y

    def lp_apply(self, v):
        """Preconditioner applied to a moment vector v [nm * NENK] (current cross sections)."""
        v = as_f64(v).ravel()
        z = np.zeros_like(v)
        self._h.call("lb_lp_apply", dptr(v), dptr(z))
        return z

    def lp_loss_grad(self, x, t, w=None):
        x = _lib.as_f32(x).reshape(-1, self.NIN)
        t = _lib.as_f32(t).reshape(-1, self.NOUT)
        wp = None if w is None else _lib.fptr(_lib.as_f32(w).ravel())
        loss = np.zeros(1)
        g = np.zeros(self.lp_nparams(), dtype=np.float32)
        self._h.call("lb_lp_loss_grad", int(x.shape[0]), _lib.fptr(x), _lib.fptr(t), wp, dptr(loss), _lib.fptr(g))
        return float(loss[0]), g

    def lp_generate(self, samples_per_group=2000, iters=8, seed=0):
        """Append (residual, error) cell samples from plain-solver runs of the problem set on this
        operator (MultigroupSolver); returns the size of the training set."""
        n = np.zeros(1, dtype=np.int64)
        self._h.call("lb_lp_generate", int(samples_per_group), int(iters), int(seed), n.ctypes.data_as(_lib._c_ll_p))
        return int(n[0])

    def lp_num_samples(self):
        n = np.zeros(1, dtype=np.int64)
        self._h.call("lb_lp_num_samples", n.ctypes.data_as(_lib._c_ll_p))
        return int(n[0])

    def lp_samples(self):
        """(features [n, 19], targets [n, 16], loss weights [n]) of the training set."""
        n = self.lp_num_samples()
        x = np.zeros((n, self.NIN), dtype=np.float32)
        t = np.zeros((n, self.NOUT), dtype=np.float32)
        w = np.zeros(n, dtype=np.float32)
        self._h.call("lb_lp_get_samples", _lib.fptr(x), _lib.fptr(t), _lib.fptr(w))
        return x, t, w

    def lp_clear(self):
        self._h.call("lb_lp_clear_samples")

    def lp_calibrate(self, m=20, rtol=1e-6):
        """(plain GMRES, learned FGMRES) operator applications per group on the current multigroup
        problem (MultigroupSolver); a held-out problem's counts decide lp_set_groups."""
        G = self.prob.G
        plain = np.zeros(G, dtype=np.int32)
        learned = np.zeros(G, dtype=np.int32)
        self._h.call("lb_lp_calibrate", int(m), float(rtol), iptr(plain), iptr(learned))
        return plain, learned

    def lp_set_groups(self, enabled=None, budget=None):
        """Groups where solver="FGMRES_ML" uses the network (None: all) and per-group caps on its
        operator applications before plain GMRES takes over (None: 4m)."""
        if enabled is None:
            self._h.call("lb_lp_set_groups", 0, None, None)
            return self
        en = np.ascontiguousarray(np.asarray(enabled, dtype=np.int32))
        bd = None if budget is None else np.ascontiguousarray(np.asarray(budget, dtype=np.int32))
        self._h.call("lb_lp_set_groups", int(en.size), iptr(en), None if bd is None else iptr(bd))
        return self

    def lp_train(self, steps=1500, batch=2048, lr=3e-3, seed=0):
        """Adam on the device-resident training set; returns the batch loss of every step."""
        hist = np.zeros(max(int(steps), 1))
        self._h.call("lb_lp_train", int(steps), int(batch), float(lr), int(seed), dptr(hist))
        return hist[:steps]

    def Destroy(self):
        self._h.close()


class TransportOp(_Op):
    name = "Transport Operator"

    def MatInv(self, s):
        """s <- T^{-1} s (TransportOperator.f90:72-151)."""
        self._h.call("lb_transport_inv", dptr(self._vec(s)))
        return s

    def MatVec(self, x):
        raise _lib.LionboltError(_lib.LB_ERR_STATE,
                                 "TransportOp%MatVec was called, but the operator has yet to be implemented.")


class ScatteringOp(_Op):
    name = "Scattering Operator"

    def MatVec(self, x):
        """x <- K x (ScatteringOperator.f90:39-70)."""
        self._h.call("lb_scatter_apply", dptr(self._vec(x)))
        return x

    def MatInv(self, s):
        raise _lib.LionboltError(_lib.LB_ERR_STATE, "ScatteringOp%MatInv was called, but this operation is undefined.")


class BoltzmannOp(_Op):
    name = "Boltzmann Operator"
    _SOLVERS = {"SI": _lib.SOLVER_SI, "GMRES": _lib.SOLVER_GMRES, "FGMRES_ML": _lib.SOLVER_FGMRES_ML,
                "FGMRES": _lib.SOLVER_FGMRES}

    def __init__(self, device=0, m=10, rtol=1e-8, atol=1e-12, maxit=0):
        super().__init__(device)
        self.m, self.rtol, self.atol, self.maxit = m, rtol, atol, maxit
        self.iters = 0
        self.resid = 0.0

    def set_right_precond_diag(self, d=None):
        """Right preconditioner of solver="FGMRES": z_j = d[j] v_j per moment row (None: identity)."""
        if d is None:
            self._h.call("lb_set_right_precond_diag", 0, None)
        else:
            d = as_f64(d).ravel()
            self._pdiag = d
            self._h.call("lb_set_right_precond_diag", int(d.size), dptr(d))
        return self

    def MatVec(self, x):
        """x <- x - T^{-1} K x (BoltzmannOperator.f90:59-104)."""
        self._h.call("lb_boltzmann_matvec", dptr(self._vec(x)))
        return x

    def MatInv(self, s, solver=None):
        """s <- L^{-1} s (BoltzmannOperator.f90:106-151).  Default solver: angular%solver."""
        solver = solver or (self.angular.solver if self.angular is not None else "GMRES")
        it = np.zeros(1, dtype=np.int32)
        rs = np.zeros(1)
        self._h.call("lb_boltzmann_solve", dptr(self._vec(s)), self._SOLVERS[solver], int(self.m), float(self.rtol),
                     float(self.atol), int(self.maxit), iptr(it), dptr(rs))
        self.iters, self.resid = int(it[0]), float(rs[0])
        return s


class MultigroupSolver(_Op):
    """Group loop of Main.f90:326-476 with the dose tally (CalculateDeposition, Main.f90:750-824)."""

    name = "Multigroup solve"

    def set_problem(self, prob):
        self.Build(prob.mesh, AngularClass(k=prob.k, w=prob.w))
        self.prob = prob
        self._h.call("lb_mg_set_problem", int(prob.G), int(prob.Ls), dptr(as_f64(prob.sigt)), dptr(as_f64(prob.sigs)),
                     dptr(as_f64(prob.dd)), dptr(as_f64(prob.unc)), dptr(as_f64(prob.beam_dir)))
        return self

    def solve(self, solver="GMRES", m=20, rtol=1e-6, atol=0.0, maxit=0):
        it = np.zeros(self.prob.G, dtype=np.int32)
        self._h.call("lb_mg_solve", BoltzmannOp._SOLVERS[solver], int(m), float(rtol), float(atol), int(maxit), iptr(it))
        return it

    def results(self):
        G, NENK = self.prob.G, self.mesh.NENK
        flux = np.zeros((G, NENK))
        dose = np.zeros(NENK)
        self._h.call("lb_mg_get_results", dptr(flux), dptr(dose))
        return flux, dose

    def write_results(self, path, particle="photon", energy_grid=None, uncollided=True, problem_type="general"):
        """Results file of the last solve in the reference's layout (LionboltHDF5.f90, Main.f90:118-231,
        :449-469, :807-821): the mesh, the particle group with its energy grid, ordinates and per-group
        fluence (and the beam's uncollided fluence in group 1), the dose deposition in the root."""
        from . import lionbolt_hdf5
        flux, dose = self.results()
        unc = None
        if uncollided and np.any(self.prob.unc):
            unc = np.zeros_like(flux)
            unc[0] = self.prob.unc
        E = energy_grid if energy_grid is not None else self.prob.energy
        return lionbolt_hdf5.write_results(path, self.mesh, self.prob.w, self.prob.k, flux, dose, particle=particle,
                                           energy_grid=E, uncollided=unc, problem_type=problem_type)


class BatchSolver:
    """Many independent multigroup dose problems solved together on one GPU (lb_batch_* C ABI):
    one persistent sweep launch over every (problem, direction) pair, lock-step GMRES with a
    device-side activity mask, and the Arnoldi matrix-vector product replayed from a CUDA graph."""

    def __init__(self, device=0):
        self.lib = _lib.load()
        b = _lib._vp()
        st = self.lib.lb_batch_create(int(device), ctypes.byref(b))
        if st != _lib.LB_OK:
            raise _lib.LionboltError(st, "lb_batch_create failed: " + self.lib.lb_status_string(st).decode())
        self.b = b
        self.problems = []

    def _check(self, st):
        if st != _lib.LB_OK:
            buf = ctypes.create_string_buffer(512)
            self.lib.lb_batch_last_error(self.b, buf, 512)
            raise _lib.LionboltError(st, buf.value.decode() or self.lib.lb_status_string(st).decode())

    def add_problem(self, prob):
        m = prob.mesh
        pid = ctypes.c_int(-1)
        self._check(self.lib.lb_batch_add_problem(
            self.b, m.NE, m.NN, dptr(as_f64(m.rg)), iptr(as_i32(m.node)), iptr(as_i32(m.neighbors)),
            iptr(as_i32(m.mat)), int(m.Nm), int(prob.k.shape[0]), dptr(as_f64(prob.k)), dptr(as_f64(prob.w)),
            int(prob.G), int(prob.Ls), dptr(as_f64(prob.sigt)), dptr(as_f64(prob.sigs)), dptr(as_f64(prob.dd)),
            dptr(as_f64(prob.unc)), dptr(as_f64(prob.beam_dir)), ctypes.byref(pid)))
        self.problems.append(prob)
        return pid.value

    def solve(self, m=20, rtol=1e-6, atol=0.0, maxit=0):
        """Operator applications per problem and group, [P, Gmax] (0 where a problem has no group)."""
        Gmax = max(p.G for p in self.problems)
        it = np.zeros((len(self.problems), Gmax), dtype=np.int32)
        self._check(self.lib.lb_batch_solve(self.b, int(m), float(rtol), float(atol), int(maxit), iptr(it)))
        return it

    def results(self, pid):
        prob = self.problems[pid]
        flux = np.zeros((prob.G, prob.mesh.NENK))
        dose = np.zeros(prob.mesh.NENK)
        self._check(self.lib.lb_batch_get_results(self.b, int(pid), dptr(flux), dptr(dose)))
        return flux, dose

    def info(self):
        n, g, th = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        ms = ctypes.c_double()
        gl, sl = ctypes.c_longlong(), ctypes.c_longlong()
        self._check(self.lib.lb_batch_info(self.b, ctypes.byref(n), ctypes.byref(g), ctypes.byref(ms), ctypes.byref(th),
                                           ctypes.byref(gl), ctypes.byref(sl)))
        return dict(problems=n.value, max_groups=g.value, last_ms=ms.value, sweep_threads=th.value,
                    graph_launches=gl.value, sweep_launches=sl.value)

    def close(self):
        if self.b:
            self.lib.lb_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
