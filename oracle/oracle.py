"""ctypes wrapper of the FP64 CPU oracle (oracle/liboracle.so) -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this module.  The oracle
restates the reference Lionbolt algorithms (see oracle.cpp for the file:line of each function);
its parity pins are the ordinate tables of the reference run logs (tests/golden/) and the closed
forms of the reference's ScatterMMS / TransportMMS drivers.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_L = ctypes.POINTER(ctypes.c_long)
_V = ctypes.c_void_p

_SIG = {
    "or_set_threads": (None, [ctypes.c_int]),
    "or_get_threads": (ctypes.c_int, []),
    "or_gauss_legendre": (None, [ctypes.c_int, _D, _D]),
    "or_sn_quadrature": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _D, _D]),
    "or_yy": (None, [ctypes.c_int, _D, _D, ctypes.c_int, _D]),
    "or_real_sh": (None, [ctypes.c_int, _D, _D]),
    "or_create": (_V, [ctypes.c_int, ctypes.c_int, _D, _I, _I, _I, ctypes.c_int]),
    "or_destroy": (None, [_V]),
    "or_nenk": (ctypes.c_long, [_V]),
    "or_get_geometry": (None, [_V, _D, _D, _D, _D, _D, _D, _D]),
    "or_set_angular": (ctypes.c_int, [_V, ctypes.c_int, _D, _D, ctypes.c_int, ctypes.c_int]),
    "or_nz": (ctypes.c_long, [_V]),
    "or_get_schedule": (None, [_V, _I, _I, _L, _L, _I, _L, _I]),
    "or_set_xs": (ctypes.c_int, [_V, _D, _D]),
    "or_transport_inv": (ctypes.c_int, [_V, _D]),
    "or_scatter_apply": (ctypes.c_int, [_V, _D]),
    "or_boltzmann_matvec": (ctypes.c_int, [_V, _D]),
    "or_boltzmann_solve": (ctypes.c_int, [_V, _D, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_int, _I, _D, _D, ctypes.c_int, _I]),
    "or_fluence": (None, [_V, _D, _D]),
    "or_multigroup": (ctypes.c_int, [_V, ctypes.c_int, _D, _D, _D, _D, _D, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_double, ctypes.c_double, ctypes.c_int, _D, _D, _I]),
    "or_set_angular_streamed": (ctypes.c_int, [_V, ctypes.c_int, _D, _D]),
    "or_set_blas": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p]),
    "or_beam_uncollided": (ctypes.c_int, [_V, _D, _D, _D, _D, ctypes.c_double, ctypes.c_double, _D, _D]),
    "or_scatter_apply_dgemv": (ctypes.c_int, [_V, _D, ctypes.c_long, ctypes.c_long]),
    "or_set_sigt": (ctypes.c_int, [_V, _D]),
    "or_moment_transport": (ctypes.c_int, [_V, ctypes.c_int, _D, _D, _D, _D]),
    "or_moment_apply": (ctypes.c_int, [_V, ctypes.c_int, _D, _D, _D]),
    "or_moment_solve": (ctypes.c_int, [_V, ctypes.c_int, _D, _D, _D, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_int, _D, _D, _D, _I, _D, _D, ctypes.c_int, _I]),
    "or_mg_moment": (ctypes.c_int, [_V, ctypes.c_int, ctypes.c_int, _D, _D, _D, _D, _D, ctypes.c_int, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_double, ctypes.c_int, _D, _D, _I, _D, _D, _I,
                                    ctypes.c_int]),
}

_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(os.path.join(HERE, "oracle.cpp")):
            build()
        lib = ctypes.CDLL(LIB)
        for n, (r, a) in _SIG.items():
            f = getattr(lib, n)
            f.restype = r
            f.argtypes = a
        _lib = lib
    return _lib


def _d(a):
    return a.ctypes.data_as(_D)


def _i(a):
    return a.ctypes.data_as(_I)


def _dn(a):
    """Pointer to a float64 array, or NULL for None."""
    return None if a is None else a.ctypes.data_as(_D)


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def sn_quadrature(Ng, Nc):
    lib = load()
    k = np.zeros((Ng * Nc, 3))
    w = np.zeros(Ng * Nc)
    lib.or_sn_quadrature(Ng, Nc, _d(k), _d(w))
    return k, w


def gauss_legendre(n):
    lib = load()
    x = np.zeros(n)
    w = np.zeros(n)
    lib.or_gauss_legendre(n, _d(x), _d(w))
    return x, w


def yy(k, w, L):
    lib = load()
    NI = k.shape[0]
    out = np.zeros((L + 1, NI, NI))
    lib.or_yy(NI, _d(np.ascontiguousarray(k)), _d(np.ascontiguousarray(w)), L, _d(out))
    return out


def real_sh(Ls, d):
    lib = load()
    Y = np.zeros((Ls + 1) ** 2)
    lib.or_real_sh(Ls, _d(np.ascontiguousarray(d, dtype=np.float64)), _d(Y))
    return Y


def set_threads(n):
    load().or_set_threads(int(n))


_blas = None


def set_blas():
    """Loads the OpenBLAS bundled with scipy (its cblas_dgemv) for Oracle.scatter_apply_dgemv, each
    OpenMP thread calling it single-threaded.  Returns the library path."""
    global _blas
    if _blas is None:
        import glob
        import scipy
        libs = sorted(glob.glob(os.path.join(os.path.dirname(scipy.__file__), os.pardir, "scipy.libs",
                                             "libscipy_openblas*.so*")))
        if not libs:
            raise RuntimeError("scipy's bundled OpenBLAS was not found")
        path = os.path.realpath(libs[0])
        if load().or_set_blas(path.encode(), b"scipy_cblas_dgemv", b"scipy_openblas_set_num_threads") != 0:
            raise RuntimeError(f"{path}: scipy_cblas_dgemv not found")
        _blas = path
    return _blas


class Oracle:
    """Literal FP64 restatement of TransportOp / ScatteringOp / BoltzmannOp."""

    def __init__(self, mesh):
        self.lib = load()
        self.mesh = mesh
        self._keep = [np.ascontiguousarray(mesh.rg, dtype=np.float64), np.ascontiguousarray(mesh.node, dtype=np.int32),
                      np.ascontiguousarray(mesh.neighbors, dtype=np.int32), np.ascontiguousarray(mesh.mat, dtype=np.int32)]
        rg, nd, nb, mt = self._keep
        self.h = self.lib.or_create(mesh.NE, mesh.NN, _d(rg), _i(nd), _i(nb), _i(mt), int(mesh.Nm))
        self.NE = mesh.NE
        self.NENK = 4 * mesh.NE
        self.NI = 0
        self.L = 0

    def close(self):
        if self.h:
            self.lib.or_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def geometry(self):
        NE = self.NE
        n = np.zeros((NE, 4, 3))
        area = np.zeros((NE, 4))
        vol = np.zeros(NE)
        detJ = np.zeros(NE)
        IC = np.zeros((NE, 3, 4, 4))
        IFM = np.zeros((NE, 4, 4, 4))
        IIM = np.zeros((NE, 4, 4, 4))
        self.lib.or_get_geometry(self.h, _d(n), _d(area), _d(vol), _d(detJ), _d(IC), _d(IFM), _d(IIM))
        # arrays are [..][kp][k] (Fortran IC(k,kp,..)); return matrices indexed [row k][col kp]
        return dict(n=n, area=area, vol=vol, detJ=detJ, IC=IC.swapaxes(-1, -2), IFM=IFM.swapaxes(-1, -2),
                    IIM=IIM.swapaxes(-1, -2))

    def set_angular(self, k, w, L, literal=True):
        self.k = np.ascontiguousarray(k, dtype=np.float64)
        self.w = np.ascontiguousarray(w, dtype=np.float64)
        self.NI = self.k.shape[0]
        self.L = L
        return self.lib.or_set_angular(self.h, self.NI, _d(self.k), _d(self.w), int(L), 1 if literal else 0)

    def schedule(self):
        NE, NI = self.NE, self.NI
        NZ = self.lib.or_nz(self.h)
        sl = np.zeros((NI, NE), dtype=np.int32)
        isl = np.zeros((NI, NE), dtype=np.int32)
        SA = np.zeros((NI, NE + 1), dtype=np.int64)
        UF = np.zeros((NI, NE + 1), dtype=np.int64)
        upf = np.zeros(NZ, dtype=np.int32)
        ipsf = np.zeros(NZ, dtype=np.int64)
        nl = np.zeros(NI, dtype=np.int32)
        self.lib.or_get_schedule(self.h, _i(sl), _i(isl), SA.ctypes.data_as(_L), UF.ctypes.data_as(_L), _i(upf),
                                 ipsf.ctypes.data_as(_L), _i(nl))
        return dict(sl=sl, isl=isl, SAoffset=SA, UFoffset=UF, upfaces=upf, ipsf=ipsf, nlevels=nl, NZ=NZ)

    def level_sets(self):
        """(sl [NI, NE], nlevels [NI]) of the current quadrature (SweepOrder.f90 sl and level counts)."""
        sl = np.zeros((self.NI, self.NE), dtype=np.int32)
        nl = np.zeros(self.NI, dtype=np.int32)
        self.lib.or_get_schedule(self.h, _i(sl), None, None, None, None, None, _i(nl))
        return sl, nl

    def set_xs(self, sigt, sigs):
        """sigt [Nm], sigs [Nm, L+1] (padded with zeros up to the angular L)."""
        sigt = np.ascontiguousarray(np.atleast_1d(sigt), dtype=np.float64)
        s = np.zeros((self.mesh.Nm, self.L + 1))
        sigs = np.atleast_2d(sigs)
        s[:, :min(sigs.shape[1], self.L + 1)] = sigs[:, :self.L + 1]
        self._xs = (sigt, np.ascontiguousarray(s))
        return self.lib.or_set_xs(self.h, _d(self._xs[0]), _d(self._xs[1]))

    def transport_inv(self, s, inplace=False):
        if inplace:
            assert s.dtype == np.float64 and s.flags.c_contiguous
        else:
            s = np.ascontiguousarray(s, dtype=np.float64).copy()
        self.lib.or_transport_inv(self.h, _d(s))
        return s

    def scatter_apply(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64).copy()
        self.lib.or_scatter_apply(self.h, _d(x))
        return x

    def set_angular_no_schedule(self, k, w, L):
        """Quadrature and YY only (no sweep schedule): enough for the scattering operator."""
        self.k = np.ascontiguousarray(k, dtype=np.float64)
        self.w = np.ascontiguousarray(w, dtype=np.float64)
        self.NI = self.k.shape[0]
        self.L = L
        return self.lib.or_set_angular(self.h, self.NI, _d(self.k), _d(self.w), int(L), 2)

    def scatter_apply_dgemv(self, x, sd0=0, sd1=None, inplace=False):
        """K x through the reference's per-node dgemv path (ScatteringAlgebra.f90:39-48, BLAS dgemv)
        on the nodes [sd0, sd1); other nodes keep their input values."""
        set_blas()
        if inplace:
            assert x.dtype == np.float64 and x.flags.c_contiguous
        else:
            x = np.ascontiguousarray(x, dtype=np.float64).copy()
        sd1 = self.NENK if sd1 is None else sd1
        st = self.lib.or_scatter_apply_dgemv(self.h, _d(x), int(sd0), int(sd1))
        if st:
            raise RuntimeError(f"or_scatter_apply_dgemv: status {st}")
        return x

    def boltzmann_matvec(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64).copy()
        self.lib.or_boltzmann_matvec(self.h, _d(x))
        return x

    def boltzmann_solve(self, s, solver="GMRES", m=10, rtol=1e-8, atol=1e-12, maxit=0):
        s = np.ascontiguousarray(s, dtype=np.float64).copy()
        it = np.zeros(1, dtype=np.int32)
        rs = np.zeros(1)
        hist = np.zeros(4096)
        hn = np.zeros(1, dtype=np.int32)
        st = self.lib.or_boltzmann_solve(self.h, _d(s), 0 if solver == "SI" else 1, int(m), float(rtol), float(atol),
                                         int(maxit), _i(it), _d(rs), _d(hist), 4096, _i(hn))
        return s, dict(status=st, iters=int(it[0]), resid=float(rs[0]), history=hist[:min(int(hn[0]), 4096)])

    def fluence(self, v):
        fl = np.zeros(self.NENK)
        self.lib.or_fluence(self.h, _d(np.ascontiguousarray(v, dtype=np.float64)), _d(fl))
        return fl

    def multigroup(self, prob, solver="GMRES", m=20, rtol=1e-10, atol=0.0, maxit=0):
        """Angular-space FP64 group loop; returns (flux [G, NENK], dose [NENK], iters [G])."""
        G, Nm = prob.G, prob.mesh.Nm
        L = self.L
        sigs = np.zeros((G, G, Nm, L + 1))
        sigs[..., :min(L, prob.Ls) + 1] = prob.sigs[..., :min(L, prob.Ls) + 1]
        args = [np.ascontiguousarray(a, dtype=np.float64) for a in (prob.sigt, sigs, prob.dd, prob.unc, prob.beam_dir)]
        flux = np.zeros((G, self.NENK))
        dose = np.zeros(self.NENK)
        it = np.zeros(G, dtype=np.int32)
        st = self.lib.or_multigroup(self.h, G, _d(args[0]), _d(args[1]), _d(args[2]), _d(args[3]), _d(args[4]),
                                    0 if solver == "SI" else 1, int(m), float(rtol), float(atol), int(maxit), _d(flux),
                                    _d(dose), _i(it))
        if st != 0:
            raise RuntimeError(f"oracle multigroup failed with status {st}")
        return flux, dose, it

    # ---- moment-space restatement (for problems whose angular Krylov space does not fit) -------------
    def set_angular_streamed(self, k, w):
        """Level sets only (no sweep-ordered offset arrays, no YY): enough for the moment-space calls."""
        self.k = np.ascontiguousarray(k, dtype=np.float64)
        self.w = np.ascontiguousarray(w, dtype=np.float64)
        self.NI = self.k.shape[0]
        self.L = 0
        return self.lib.or_set_angular_streamed(self.h, self.NI, _d(self.k), _d(self.w))

    def set_sigt(self, sigt):
        self._sigt = np.ascontiguousarray(np.atleast_1d(sigt), dtype=np.float64)
        return self.lib.or_set_sigt(self.h, _d(self._sigt))

    @staticmethod
    def _sigl(sigs, Nm, Ls):
        out = np.zeros((Nm, Ls + 1))
        sigs = np.atleast_2d(sigs)
        out[:, :min(sigs.shape[1], Ls + 1)] = sigs[:, :Ls + 1]
        return out

    def moment_transport(self, Ls, s=None, q=None, want_psi=False):
        """y = D T^-1 (M s + q) [nm, NENK] (and psi = T^-1 (M s + q) [NI * NENK] when asked)."""
        nm = (Ls + 1) ** 2
        s, q = _f64(s), _f64(q)
        y = np.zeros((nm, self.NENK))
        psi = np.zeros(self.NI * self.NENK) if want_psi else None
        st = self.lib.or_moment_transport(self.h, int(Ls), _dn(s), _dn(q), _d(y), _dn(psi))
        if st:
            raise RuntimeError(f"or_moment_transport: status {st}")
        return (y, psi) if want_psi else y

    def moment_apply(self, Ls, sigs, x):
        """A x = x - D T^-1 M S x for moment vectors x [nm, NENK]; sigs [Nm, Ls+1]."""
        sigl = self._sigl(sigs, self.mesh.Nm, Ls)
        x = _f64(x)
        y = np.zeros_like(x)
        st = self.lib.or_moment_apply(self.h, int(Ls), _d(sigl), _d(x), _d(y))
        if st:
            raise RuntimeError(f"or_moment_apply: status {st}")
        return y

    def moment_solve(self, Ls, sigs, q=None, s_mom=None, m=20, rtol=1e-10, atol=0.0, maxit=0, pdiag=None,
                     want_psi=False):
        """Within-group solve A phi = D T^-1 (q + M s_mom) from phi0 = b: GMRES(m), or FGMRES(m) with the
        right preconditioner z_j = pdiag[j] v_j.  Returns (phi [nm, NENK], psi or None, info)."""
        nm = (Ls + 1) ** 2
        sigl = self._sigl(sigs, self.mesh.Nm, Ls)
        q, s_mom, pdiag = _f64(q), _f64(s_mom), _f64(pdiag)
        phi = np.zeros((nm, self.NENK))
        psi = np.zeros(self.NI * self.NENK) if want_psi else None
        it = np.zeros(1, dtype=np.int32)
        rs = np.zeros(1)
        hist = np.zeros(4096)
        hn = np.zeros(1, dtype=np.int32)
        st = self.lib.or_moment_solve(self.h, int(Ls), _d(sigl), _dn(q), _dn(s_mom), int(m), float(rtol), float(atol),
                                      int(maxit), _dn(pdiag), _d(phi), _dn(psi), _i(it), _d(rs), _d(hist), 4096, _i(hn))
        return phi, psi, dict(status=st, iters=int(it[0]), resid=float(rs[0]), history=hist[:min(int(hn[0]), 4096)])

    def mg_moment(self, prob, m=20, rtol=1e-10, rtol_snap=0.0, atol=0.0, maxit=0, verbose=False):
        """Moment-space FP64 group loop.  Returns dict(flux [G, NENK], dose [NENK], iters [G]) and, with
        rtol_snap > rtol, flux_snap / dose_snap / iters_snap of each group first solved to rtol_snap."""
        G, Nm, Ls = prob.G, prob.mesh.Nm, prob.Ls
        args = [np.ascontiguousarray(a, dtype=np.float64) for a in (prob.sigt, prob.sigs, prob.dd, prob.unc,
                                                                    prob.beam_dir)]
        assert args[1].shape == (G, G, Nm, Ls + 1)
        flux = np.zeros((G, self.NENK))
        dose = np.zeros(self.NENK)
        it = np.zeros(G, dtype=np.int32)
        snap = rtol_snap > rtol
        fs = np.zeros((G, self.NENK)) if snap else None
        ds = np.zeros(self.NENK) if snap else None
        its = np.zeros(G, dtype=np.int32)
        st = self.lib.or_mg_moment(self.h, G, Ls, _d(args[0]), _d(args[1]), _d(args[2]), _d(args[3]), _d(args[4]),
                                   int(m), float(rtol), float(rtol_snap), float(atol), int(maxit), _d(flux), _d(dose),
                                   _i(it), _dn(fs), _dn(ds), _i(its), int(bool(verbose)))
        if st != 0:
            raise RuntimeError(f"oracle moment-space multigroup failed with status {st}")
        out = dict(flux=flux, dose=dose, iters=it)
        if snap:
            out.update(flux_snap=fs, dose_snap=ds, iters_snap=its)
        return out

    def beam_uncollided(self, origin, axis, e1, e2, w1, w2, attn):
        """Uncollided fluence of a planar rectangular beam at the DG nodes [NENK] (reference ray tracing
        against region faces, Beer's law, projection onto the DG basis)."""
        f = lambda a: np.ascontiguousarray(a, dtype=np.float64)
        args = [f(origin), f(axis), f(e1), f(e2)]
        at = f(np.atleast_1d(attn))
        unc = np.zeros(self.NENK)
        st = self.lib.or_beam_uncollided(self.h, *[_d(a) for a in args], float(w1), float(w2), _d(at), _d(unc))
        if st:
            raise RuntimeError("oracle ray tracing found no boundary intersection")
        return unc
