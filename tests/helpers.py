"""Shared helpers for the parity tests (the oracle is the checker, never the product)."""
import decimal
import fractions
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def golden(name):
    return np.loadtxt(os.path.join(GOLDEN, name))


def scatter_moment(n):
    """XS%s(n) of the reference's ScatterMMS driver (validation/operators/ScatterMMS.f90:91-128):
    2 pi (S1 e - S2 (-1)^n / e), zero for n >= 14, evaluated in extended precision."""
    if n >= 14:
        return 0.0
    S1 = fractions.Fraction(0)
    S2 = fractions.Fraction(0)
    tmp = fractions.Fraction(1)
    for m in range(n + 1):
        S1 += tmp * (-1) ** m
        S2 += tmp
        if m == n:
            break
        tmp = tmp * (n + m + 1) * (n - m) / (2 * (m + 1))
    with decimal.localcontext() as ctx:
        ctx.prec = 50
        e = decimal.Decimal(1).exp()
        d1 = decimal.Decimal(S1.numerator) / decimal.Decimal(S1.denominator)
        d2 = decimal.Decimal(S2.numerator) / decimal.Decimal(S2.denominator)
        f = d1 * e - d2 * (-1) ** n / e
    return 2.0 * np.pi * float(f)


def scatter_mms(mesh, k):
    """Input psi = exp(r.k) and exact K psi = 2 pi (e^t - e^-t)/t, t = |r + k| (ScatterMMS.f90:51-70)."""
    r = mesh.node_coords()                      # [NENK, 3]
    psi = np.exp(k @ r.T)                       # [NI, NENK]
    t = np.linalg.norm(r[None, :, :] + k[:, None, :], axis=2)
    exact = np.where(t == 0, 4 * np.pi, 2 * np.pi * (np.exp(t) - np.exp(-t)) / np.where(t == 0, 1, t))
    return psi.ravel(), exact.ravel()


def transport_mms(mesh, k, sigma=1e-10, A=10.0):
    """Source (-2A k.r + sigma) exp(-A r^2) and exact exp(-A r^2) (TransportMMS.f90:62-77)."""
    r = mesh.node_coords()
    g = np.exp(-A * (r * r).sum(axis=1))
    src = (-2 * A * (k @ r.T) + sigma) * g[None, :]
    exact = np.broadcast_to(g[None, :], src.shape)
    return src.ravel(), np.ascontiguousarray(exact).ravel()


def jittered(mesh, amount, seed=1):
    """Copy of a box mesh with interior nodes moved randomly (general face normals)."""
    rg = mesh.rg.copy()
    lo, hi = rg.min(axis=0), rg.max(axis=0)
    interior = np.all((rg > lo + 1e-12) & (rg < hi - 1e-12), axis=1)
    rng = np.random.default_rng(seed)
    rg[interior] += amount * rng.uniform(-1, 1, size=(interior.sum(), 3))
    from lionbolt_b200.mesh import Mesh
    return Mesh(rg=rg, node=mesh.node.copy(), neighbors=mesh.neighbors.copy(), mat=mesh.mat.copy(), Nm=mesh.Nm,
                shape=mesh.shape)


def golden_mesh(name):
    """A mesh of the reference's tree stored as a tests/golden fixture (make_mesh_fixtures.py):
    nodes, connectivity and materials as read by read_gmsh, neighbours rebuilt by face matching."""
    from lionbolt_b200.mesh import Mesh, neighbours
    d = np.load(os.path.join(GOLDEN, f"mesh_{name}.npz"))
    node = d["node"].astype(np.int32)
    mat = d["mat"].astype(np.int32)
    return Mesh(rg=d["rg"].astype(np.float64), node=node, neighbors=neighbours(node), mat=mat, Nm=int(mat.max()) + 1)


def layered_beam_reference(mesh, center, width, layers):
    """Uncollided fluence of a normally incident (+z) rectangular beam entering at z = 0, at the DG
    nodes, in closed form for a mesh whose materials are layers in z: exp(-tau) at the 4-point rule's
    points (barycentric a on vertex k), tau = sum_layers sigma * (length of [0, z] in the layer), then
    the L2 projection onto the linear basis c_k = sqrt(5) phi_k + (1 - sqrt(5))/4 sum_q phi_q.
    layers: list of (z0, z1, sigma)."""
    a, b = (5 + 3 * np.sqrt(5)) / 20, (5 - np.sqrt(5)) / 20
    X = mesh.rg[mesh.node]                                   # [NE, 4, 3]
    W = np.full((4, 4), b) + (a - b) * np.eye(4)             # [q, k]
    Q = np.einsum("qk,ekd->eqd", W, X)                       # [NE, 4, 3]
    inside = (np.abs(Q[..., 0] - center[0]) <= 0.5 * width[0] + 1e-12) & \
             (np.abs(Q[..., 1] - center[1]) <= 0.5 * width[1] + 1e-12)
    z = Q[..., 2]
    tau = np.zeros_like(z)
    for z0, z1, sig in layers:
        tau += sig * np.clip(np.minimum(z, z1) - z0, 0.0, None)
    phi = np.where(inside, np.exp(-tau), 0.0)
    c = np.sqrt(5) * phi + 0.25 * (1 - np.sqrt(5)) * phi.sum(axis=1, keepdims=True)
    return c.ravel()


def replica_rank(rank, world, port, out):
    """One gloo rank of the replicas path of bench.py: the max-over-ranks reduction its timings go
    through, and the reference arm, which runs on rank 0 only (the other ranks exit 0 without work)."""
    import contextlib
    import datetime
    import io
    import sys as _sys
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if root not in _sys.path:
        _sys.path.insert(0, root)
    import bench
    res = {"env": bench.dist_env(), "max": bench.rank_max(10.0 + 2.5 * rank),
           "max_neg": bench.rank_max(-1.0 - rank)}
    if rank != 0:
        buf = io.StringIO()
        with contextlib.redirect_stdout(buf):
            res["ref_rc"] = bench.run_reference(None)
        res["ref_out"] = buf.getvalue()
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, res))
