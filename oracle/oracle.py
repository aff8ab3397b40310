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

    def set_xs(self, sigt, sigs):
        """sigt [Nm], sigs [Nm, L+1] (padded with zeros up to the angular L)."""
        sigt = np.ascontiguousarray(np.atleast_1d(sigt), dtype=np.float64)
        s = np.zeros((self.mesh.Nm, self.L + 1))
        sigs = np.atleast_2d(sigs)
        s[:, :min(sigs.shape[1], self.L + 1)] = sigs[:, :self.L + 1]
        self._xs = (sigt, np.ascontiguousarray(s))
        return self.lib.or_set_xs(self.h, _d(self._xs[0]), _d(self._xs[1]))

    def transport_inv(self, s):
        s = np.ascontiguousarray(s, dtype=np.float64).copy()
        self.lib.or_transport_inv(self.h, _d(s))
        return s

    def scatter_apply(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64).copy()
        self.lib.or_scatter_apply(self.h, _d(x))
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
