"""NumPy FP64 reference of the learned preconditioner's network, features and gradients.

This is test infrastructure: it checks the CUDA inference, preconditioner and training kernels.
The forward pass reproduces the kernels' BF16 rounding points (weights, inputs and hidden
activations rounded to BF16, biases and accumulation kept wide); the backward pass treats the
rounding as identity (straight-through), like the training kernel.  With round=False everything is
plain FP64, which the finite-difference check in test_mlp_ref.py uses.
"""
import numpy as np

NIN, NH, NOUT, NMOM = 19, 64, 16, 16
OFF_W1 = 0
OFF_B1 = OFF_W1 + NH * NIN
OFF_W2 = OFF_B1 + NH
OFF_B2 = OFF_W2 + NH * NH
OFF_W3 = OFF_B2 + NH
OFF_B3 = OFF_W3 + NOUT * NH
NPARAM = OFF_B3 + NOUT


def bf16(a):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(w):
    w = np.asarray(w, dtype=np.float64)
    return (w[OFF_W1:OFF_B1].reshape(NH, NIN), w[OFF_B1:OFF_W2], w[OFF_W2:OFF_B2].reshape(NH, NH),
            w[OFF_B2:OFF_W3], w[OFF_W3:OFF_B3].reshape(NOUT, NH), w[OFF_B3:NPARAM])


def forward(w, x, round=True):
    """Outputs [n, 16] and the intermediates needed by backward()."""
    r = bf16 if round else (lambda a: np.asarray(a, dtype=np.float64))
    W1, b1, W2, b2, W3, b3 = unpack(w)
    W1, W2, W3 = r(W1), r(W2), r(W3)
    xb = r(x)
    z1 = xb @ W1.T + b1
    h1 = r(np.maximum(z1, 0.0))
    z2 = h1 @ W2.T + b2
    h2 = r(np.maximum(z2, 0.0))
    o = h2 @ W3.T + b3
    return o, (xb, z1, h1, z2, h2, W1, W2, W3)


def loss_grad(w, x, t, wts=None, round=True):
    """L = 1/(2n) sum_k wts_k |o_k - t_k|^2 and dL/dw in the flat parameter layout."""
    n = x.shape[0]
    wts = np.ones(n) if wts is None else np.asarray(wts, dtype=np.float64)
    o, (xb, z1, h1, z2, h2, W1, W2, W3) = forward(w, x, round)
    d = o - t
    loss = 0.5 * np.sum(wts[:, None] * d * d) / n
    d3 = wts[:, None] * d / n
    g = np.zeros(NPARAM)
    g[OFF_W3:OFF_B3] = (d3.T @ h2).ravel()
    g[OFF_B3:NPARAM] = d3.sum(axis=0)
    d2 = (d3 @ W3) * (z2 > 0)
    g[OFF_W2:OFF_B2] = (d2.T @ h1).ravel()
    g[OFF_B2:OFF_W3] = d2.sum(axis=0)
    d1 = (d2 @ W2) * (z1 > 0)
    g[OFF_W1:OFF_B1] = (d1.T @ xb).ravel()
    g[OFF_B1:OFF_W2] = d1.sum(axis=0)
    return loss, g


def mean_chord(mesh):
    """4V/S of every tetrahedron (Cauchy's mean chord)."""
    p = mesh.rg[mesh.node]                                   # [NE, 4, 3]
    vol = np.abs(np.einsum("ij,ij->i", np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), p[:, 3] - p[:, 0])) / 6
    faces = [(0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3)]
    S = sum(0.5 * np.linalg.norm(np.cross(p[:, b] - p[:, a], p[:, c] - p[:, a]), axis=1) for a, b, c in faces)
    return 4 * vol / S


def features(v, mesh, sigt, sigs0, nm):
    """Per-cell network inputs [NE, 19] and scales [NE] of a moment vector v [nm * NENK]."""
    NE = mesh.NE
    nmom = min(nm, NMOM)
    V = np.asarray(v, dtype=np.float64).reshape(nm, NE, 4)
    avg = np.zeros((NE, NMOM))
    avg[:, :nmom] = V[:nmom].mean(axis=2).T
    s = np.sqrt((avg ** 2).sum(axis=1) / nmom)
    inv = np.where(s > 0, 1.0 / np.where(s > 0, s, 1.0), 0.0)
    x = np.zeros((NE, NIN))
    x[:, :NMOM] = avg * inv[:, None]
    ell = mean_chord(mesh)
    st = np.asarray(sigt, dtype=np.float64)[mesh.mat]
    ss = np.asarray(sigs0, dtype=np.float64)[mesh.mat]
    x[:, 16] = st * ell
    x[:, 17] = ss * ell
    x[:, 18] = np.where(st > 0, ss / np.where(st > 0, st, 1.0), 0.0)
    return x, s


def apply(w, v, mesh, sigt, sigs0, nm):
    """z = v + s * net(x) on the cell's 4 nodes for moments j < 16."""
    x, s = features(v, mesh, sigt, sigs0, nm)
    o, _ = forward(w, x)
    z = np.array(v, dtype=np.float64).reshape(nm, mesh.NE, 4)
    nmom = min(nm, NMOM)
    z[:nmom] += (s[:, None] * o[:, :nmom]).T[:, :, None]
    return z.ravel()
