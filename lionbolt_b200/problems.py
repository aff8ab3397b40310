"""Seeded synthetic transport problems with the shapes of the benchmark configurations.

The reference's inputs come from gmsh meshes and the NittanyPhysics cross-section library, neither
of which is available; these builders produce the same array shapes from closed-form, seeded
definitions:

  config0  10 cm cube, 10^3 hexes x 6 = 6,000 tets, 80 directions (Ng, Nc) = (8, 10), 1 group,
           sigma_t = 0.2, c = 0.9, Henyey-Greenstein g = 0.8 truncated at P3 (16 moments),
           5 x 5 cm normally incident beam on z = 0 as a first-collision source.
  config1  20 x 20 x 40 cm, 40 x 40 x 80 hexes = 768,000 tets, 288 directions (L = 11,
           (Ng, Nc) = (12, 24)), 20 groups, P5 (36 moments), downscatter-only row-stochastic
           transfer matrix, HG g from 0.5 to 0.95, sigma_t ~ logU[0.02, 0.5] per group, a 2 cm
           aluminium-like slab (sigma x 2.7) at z in [5, 7] cm, beam 15 degrees off the z axis.

The beam is monodirectional; its uncollided flux u(r) = exp(-tau(r)) inside the beam column is
evaluated at every DG node and enters group 0 as a first-collision source (FCSSource.f90,
AddAngularFluence.f90 compute the same quantity by ray tracing).  The dose cross section is
absorption (sigma_t - sigma_s,out) times the group mid-point energy.
"""
from dataclasses import dataclass

import numpy as np

from . import mesh as _mesh


@dataclass
class Problem:
    name: str
    mesh: _mesh.Mesh
    k: np.ndarray          # [NI, 3]
    w: np.ndarray          # [NI]
    Ng: int
    Nc: int
    G: int
    Ls: int                # Legendre order of scattering
    sigt: np.ndarray       # [G, Nm]
    sigs: np.ndarray       # [G, G, Nm, Ls+1] transfer g' -> g (sigs[g, g] within group)
    dd: np.ndarray         # [G, Nm]
    unc: np.ndarray        # [NENK] uncollided scalar flux of the beam (group 0)
    beam_dir: np.ndarray   # [3]
    energy: np.ndarray = None   # [G + 1] group bounds (MeV), when the builder defines them

    @property
    def NI(self):
        return int(self.k.shape[0])

    @property
    def nm(self):
        return (self.Ls + 1) ** 2

    def within_group(self, g):
        """(sigt [Nm], sigs [Nm, Ls+1]) of group g."""
        return self.sigt[g].copy(), self.sigs[g, g].copy()


def quadrature(Ng, Nc):
    """GL x Chebyshev product quadrature, SNPrep.f90:39-76 ordering (j azimuth outer)."""
    mu, wg = np.polynomial.legendre.leggauss(Ng)
    k = np.zeros((Ng * Nc, 3))
    w = np.zeros(Ng * Nc)
    ii = 0
    for j in range(1, Nc + 1):
        phi = (2 * j - 1) * np.pi / Nc
        for i in range(Ng):
            st = np.sqrt(1.0 - mu[i] ** 2)
            k[ii] = (np.cos(phi) * st, np.sin(phi) * st, mu[i])
            w[ii] = wg[i] * 2.0 * np.pi / Nc
            ii += 1
    return k, w


def beam_uncollided(mesh, beam_dir, center, width, sigma_of_z):
    """exp(-optical depth) at every DG node inside a rectangular beam entering through z = 0.

    sigma_of_z: list of (z0, z1, sigma) layers covering the box depth.
    """
    r = mesh.node_coords()
    b = np.asarray(beam_dir, dtype=np.float64)
    b = b / np.linalg.norm(b)
    t = r[:, 2] / b[2]
    r0 = r - t[:, None] * b[None, :]
    inside = (np.abs(r0[:, 0] - center[0]) <= 0.5 * width[0]) & (np.abs(r0[:, 1] - center[1]) <= 0.5 * width[1])
    tau = np.zeros(r.shape[0])
    for z0, z1, sig in sigma_of_z:
        seg = np.clip(np.minimum(r[:, 2], z1) - z0, 0.0, None)
        tau += sig * seg / b[2]
    return np.where(inside, np.exp(-tau), 0.0)


def config0():
    m = _mesh.box_mesh(10, 10, 10, (0, 0, 0), (10, 10, 10))
    Ng, Nc = 8, 10
    k, w = quadrature(Ng, Nc)
    Ls = 3
    sigt = np.array([[0.2]])
    c, g = 0.9, 0.8
    sigs = np.zeros((1, 1, 1, Ls + 1))
    sigs[0, 0, 0, :] = [c * 0.2 * g ** l for l in range(Ls + 1)]
    dd = np.array([[0.2 * (1 - c)]])
    bdir = np.array([0.0, 0.0, 1.0])
    unc = beam_uncollided(m, bdir, (5.0, 5.0), (5.0, 5.0), [(0.0, 10.0, 0.2)])
    return Problem("config0", m, k, w, Ng, Nc, 1, Ls, sigt, sigs, dd, unc, bdir)


def multigroup_box(n=(40, 40, 80), size=(20.0, 20.0, 40.0), Ng=12, Nc=24, G=20, Ls=5, seed=20261203,
                   slab=(5.0, 7.0), slab_scale=2.7, beam_deg=15.0, beam_width=(5.0, 5.0), name="config1"):
    """config1 when called with defaults; smaller meshes / fewer groups keep the same physics."""
    nx, ny, nz = n
    sx, sy, sz = size

    def material(cent):
        return ((cent[:, 2] >= slab[0]) & (cent[:, 2] <= slab[1])).astype(np.int32)

    m = _mesh.box_mesh(nx, ny, nz, (0, 0, 0), (sx, sy, sz), material=material, Nm=2)
    k, w = quadrature(Ng, Nc)
    rng = np.random.default_rng(seed)
    st_water = np.exp(rng.uniform(np.log(0.02), np.log(0.5), size=G))
    sigt = np.stack([st_water, slab_scale * st_water], axis=1)                 # [G, 2]
    # downscatter-only, row-stochastic transfer probabilities P[g, g'] (g' >= g)
    P = np.triu(rng.uniform(0.0, 1.0, size=(G, G)))
    P[np.arange(G), np.arange(G)] += 1.0                                      # favour self-scatter
    P /= P.sum(axis=1, keepdims=True)
    hg = np.linspace(0.5, 0.95, G)
    sigs = np.zeros((G, G, 2, Ls + 1))
    for gp in range(G):
        for g in range(gp, G):
            for mm in range(2):
                sigs[gp, g, mm, :] = 0.9 * sigt[gp, mm] * P[gp, g] * hg[gp] ** np.arange(Ls + 1)
    energy = np.geomspace(6.0, 0.01, G + 1)
    emid = 0.5 * (energy[:-1] + energy[1:])
    dd = np.zeros((G, 2))
    for g in range(G):
        for mm in range(2):
            dd[g, mm] = (sigt[g, mm] - sigs[g, :, mm, 0].sum()) * emid[g]
    th = np.deg2rad(beam_deg)
    bdir = np.array([np.sin(th), 0.0, np.cos(th)])
    layers = [(0.0, slab[0], st_water[0]), (slab[0], slab[1], slab_scale * st_water[0]), (slab[1], sz, st_water[0])]
    unc = beam_uncollided(m, bdir, (0.5 * sx, 0.5 * sy), beam_width, layers)
    return Problem(name, m, k, w, Ng, Nc, G, Ls, sigt, sigs, dd, unc, bdir, energy)


def config1():
    return multigroup_box()


def config1_small(n=(8, 8, 16), G=4, Ng=6, Nc=12):
    """config1 physics on a coarse mesh with fewer groups and directions (oracle-sized)."""
    return multigroup_box(n=n, G=G, Ng=Ng, Nc=Nc, name=f"config1_small{n}")


SN_ORDERS = {8: (8, 10), 12: (12, 14), 16: (16, 18)}   # S_N -> (polar Ng, azimuthal Nc): N(N+2) directions


def batch_problem(rng, idx, hmin=8, hmax=32, cell=0.5, groups=(1, 10), orders=(8, 12, 16), Ls=3):
    """One problem of a batched workload: hexes per axis ~ U{hmin..hmax} (x6 tets), S_N mixed,
    1-10 groups, P3, cross sections drawn like config1 (log-uniform water + a slab x2.7), beam
    direction uniform on the upper hemisphere and width U[1, 8] cm."""
    n = tuple(int(v) for v in rng.integers(hmin, hmax + 1, size=3))
    size = tuple(cell * v for v in n)
    G = int(rng.integers(groups[0], groups[1] + 1))
    N = int(rng.choice(orders))
    Ng, Nc = SN_ORDERS[N]
    depth = size[2]
    z0 = float(rng.uniform(0.15, 0.6)) * depth
    slab = (z0, min(depth, z0 + 0.1 * depth))
    u = rng.uniform(0.0, 1.0)                      # uniform on the upper hemisphere: cos(theta) ~ U[0, 1]
    ct = max(u, 0.05)
    ph = rng.uniform(0.0, 2 * np.pi)
    st = np.sqrt(1 - ct * ct)
    width = float(rng.uniform(1.0, 8.0))
    seed = int(rng.integers(0, 2 ** 31 - 1))
    prob = multigroup_box(n=n, size=size, Ng=Ng, Nc=Nc, G=G, Ls=Ls, seed=seed, slab=slab,
                          beam_deg=0.0, name=f"batch{idx}")
    bdir = np.array([st * np.cos(ph), st * np.sin(ph), ct])
    layers = [(0.0, slab[0], prob.sigt[0, 0]), (slab[0], slab[1], prob.sigt[0, 1]), (slab[1], depth, prob.sigt[0, 0])]
    beam = (min(width, size[0]), min(width, size[1]))
    prob.beam_dir = bdir
    prob.unc = beam_uncollided(prob.mesh, bdir, (0.5 * size[0], 0.5 * size[1]), beam, layers)
    return prob


def batch_problems(count=64, seed=20261203, **kw):
    """config3: `count` independent problems with seeded uneven sizes (8^3 to 32^3 hexes)."""
    rng = np.random.default_rng(seed)
    return [batch_problem(rng, i, **kw) for i in range(count)]
