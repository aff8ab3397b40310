"""Regenerates tests/golden/config1_oracle.npz: the FP64 oracle's solution of the 768,000-tet,
288-direction, 20-group dose problem (lionbolt_b200.problems.config1), which is too large to keep
whole in the repository or to recompute inside a test.

The oracle is the moment-space FP64 restatement (oracle/oracle.cpp, MomentSpace / or_mg_moment):
per group GMRES(20) in flux-moment space with literal per-direction sweeps streamed in batches,
every group solved to a relative residual of 1e-10 (the converged FP64 answer).  Each group is first
solved to 1e-6 and that iterate continued, so the fixture also records how far a 1e-6 solve is from
the converged one in FP64 (snap_*).  Stored:

  nodes          [4096]      seeded sample of DG node indices (sorted)
  flux, dose     [20][4096], [4096]  scalar fluence per group and dose at those nodes
  flux_norm      [20]        L2 norm of each group's fluence over all 3,072,000 nodes
  dose_norm      []          L2 norm of the dose over all nodes
  flux_layers    [20][80]    sum of each group's fluence over the DG nodes of each hex layer along z
  dose_layers    [80]        the same for the dose (every node enters one layer sum)
  snap_flux_rel_l2 [20], snap_dose_rel_l2   rel. L2 (all nodes) of the 1e-6 solve vs the 1e-10 solve
  iters, iters_snap [20]     operator applications per group (total, and of the 1e-6 part)
  nlevels        [288]       wavefront levels per direction (SweepOrder.f90 level sets)
  sl_sha256                  SHA-256 of the level-set element order sl [288][768000] (int32, little endian)
  meta                       JSON: tolerances, thread count, CPU, wall time, command

Run (about 75 minutes on 8 cores, 45 GB of host memory):
  python tests/golden/make_config1_fixture.py [--threads N]
"""
import argparse
import hashlib
import json
import os
import platform
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402
from lionbolt_b200 import problems as P  # noqa: E402

SAMPLE = 4096
SAMPLE_SEED = 20261204


def layer_sums(v, shape):
    """Sum of a per-DG-node field over each hex layer along z of a box mesh (6 tets per hex)."""
    nx, ny, nz = shape
    return v.reshape(nz, nx * ny * 6 * 4).sum(axis=1)


def summarise(flux, dose, shape, nodes):
    return dict(flux=flux[:, nodes], dose=dose[nodes], flux_norm=np.linalg.norm(flux, axis=1),
                dose_norm=np.linalg.norm(dose), flux_layers=np.stack([layer_sums(f, shape) for f in flux]),
                dose_layers=layer_sums(dose, shape))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count())
    ap.add_argument("--rtol", type=float, default=1e-10)
    ap.add_argument("--rtol-snap", type=float, default=1e-6)
    ap.add_argument("--out", default=os.path.join(HERE, "config1_oracle.npz"))
    args = ap.parse_args()
    O.set_threads(args.threads)
    t0 = time.time()
    prob = P.config1()
    m = prob.mesh
    o = O.Oracle(m)
    assert o.set_angular_streamed(prob.k, prob.w) == 0
    sl, nl = o.level_sets()
    sl_hash = hashlib.sha256(np.ascontiguousarray(sl, dtype="<i4").tobytes()).hexdigest()
    del sl
    print(f"schedule: {time.time() - t0:.1f} s, levels {nl.min()}..{nl.max()}", flush=True)
    r = o.mg_moment(prob, m=20, rtol=args.rtol, rtol_snap=args.rtol_snap, verbose=True)
    wall = time.time() - t0
    rng = np.random.default_rng(SAMPLE_SEED)
    nodes = np.sort(rng.choice(m.NENK, size=SAMPLE, replace=False))
    out = summarise(r["flux"], r["dose"], m.shape, nodes)
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    snap_flux = np.array([rel(r["flux_snap"][g], r["flux"][g]) for g in range(prob.G)])
    snap_dose = rel(r["dose_snap"], r["dose"])
    cpu = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            cpu = next(l.split(":", 1)[1].strip() for l in f if l.startswith("model name"))
    except (OSError, StopIteration):
        pass
    meta = dict(problem="config1: 40x40x80 hexes x 6 = 768000 tets, 288 directions (L = 11), 20 groups, P5, "
                        "2 materials, beam 15 degrees off axis (lionbolt_b200.problems.config1)",
                solver=f"moment-space FP64 GMRES(20), phi0 = b, rtol {args.rtol:g} (snapshots at "
                       f"{args.rtol_snap:g}), stopping test ||b - A phi|| <= rtol ||b||",
                threads=args.threads, cpu=cpu, host=platform.node(), wall_seconds=wall,
                command="python tests/golden/make_config1_fixture.py " + " ".join(sys.argv[1:]))
    np.savez_compressed(args.out, nodes=nodes, **out, snap_flux_rel_l2=snap_flux, snap_dose_rel_l2=snap_dose,
                        iters=r["iters"], iters_snap=r["iters_snap"], nlevels=nl, sl_sha256=sl_hash,
                        meta=json.dumps(meta))
    print(json.dumps(dict(meta, iters=r["iters"].tolist(), iters_snap=r["iters_snap"].tolist(),
                          snap_flux_rel_l2=snap_flux.tolist(), snap_dose_rel_l2=snap_dose)), flush=True)


if __name__ == "__main__":
    main()
