#!/usr/bin/env python
"""Benchmark: time-to-dose of the multigroup transport solve on B200, and the CPU baseline.

Workload (one step): the full multigroup dose solve of the 768,000-tet box (40 x 40 x 80 hexes,
20 x 20 x 40 cm, 288 directions, 20 groups, P5 scattering, 2 materials, beam 15 degrees off axis),
every group solved to a 1e-6 relative moment residual.  Synthetic, seeded inputs (no dataset).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--solver GMRES|FGMRES_ML]

value = dose solves per second over all ranks (replicas: every rank solves its own copy, so the
per-rank work is fixed and scaling is weak); ms_per_step = time-to-dose.  Device time is measured
with CUDA events on the library's stream, max over ranks.  `e2e` repeats the solve through the
public C ABI with the per-step inputs copied from pinned host memory and the dose read back.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "B200 time-to-dose @1e-6 resid: learned-precond FGMRES vs plain GMRES; sweep GB/s"
UNIT = "cell-direction-group updates/s"
NE_NI_NOTE = "an update = one element x one direction x one group of a transport sweep"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--solver", default="GMRES", choices=["GMRES", "FGMRES_ML", "SI"])
    p.add_argument("--m", type=int, default=20)
    p.add_argument("--rtol", type=float, default=1e-6)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-seconds", type=float, default=20.0)
    p.add_argument("--mesh", type=int, nargs=3, default=None, metavar=("NX", "NY", "NZ"),
                   help="hexes per axis of a reduced box with the same physics (profiling cases)")
    p.add_argument("--groups", type=int, default=None, help="energy groups of the reduced box")
    p.add_argument("--workload", default="dose", choices=["dose", "gemm", "batch", "mesh", "beam"],
                   help="dose: multigroup dose solve (default); gemm: standalone moment-to-discrete and "
                        "discrete-to-moment contractions at the 768k-tet size, split-BF16 vs cuBLAS FP32 vs FP64; "
                        "batch: 64 independent problems (8^3..32^3 hexes, S8/S12/S16, 1-10 groups, P3) solved "
                        "together; mesh: sweep throughput of a within-group solve on --mesh-file; beam: the "
                        "ray-traced first-collision data of the dose workload's beam (--mesh reduces it)")
    p.add_argument("--batch-count", type=int, default=64, help="problems of --workload batch (profiling cases)")
    p.add_argument("--mesh-file", default=os.path.join(ROOT, "tests", "golden", "mesh_het_cube_spherical_beam.npz"),
                   help="mesh of --workload mesh: .npz fixture, gmsh .msh, or 'jittered' (768k-tet box, moved nodes)")
    p.add_argument("--no-subbench", action="store_true",
                   help="skip the standalone-contraction and batched sub-records of the default line")
    p.add_argument("--no-learned", action="store_true",
                   help="skip the learned-preconditioner FGMRES comparison (training + timed solves)")
    p.add_argument("--lp-problems", type=int, default=3, help="training problems (seeded cross sections / slab)")
    p.add_argument("--lp-samples", type=int, default=2000, help="training samples per group and problem")
    p.add_argument("--lp-steps", type=int, default=1500, help="Adam steps")
    p.add_argument("--profile-range", action="store_true",
                   help="bracket the device-timed steps with cudaProfilerStart/Stop (ncu --profile-from-start off)")
    return p.parse_args()


def workload(args):
    """The benchmarked problem: config1 (768,000 tets, 288 directions, 20 groups) unless reduced."""
    from lionbolt_b200 import problems as P
    full, wl = workload_name(args)
    if full:
        return P.config1(), wl
    n = tuple(args.mesh) if args.mesh else (40, 40, 80)
    G = args.groups or 20
    prob = P.multigroup_box(n=n, size=(0.5 * n[0], 0.5 * n[1], 0.5 * n[2]), G=G,
                            slab=(5.0 * n[2] / 80, 7.0 * n[2] / 80), name=f"box{n}")
    return prob, wl


def bench_config(args, world):
    """The workload description both arms print (the reference arm times a slice of the same problem)."""
    _, wl = workload_name(args)
    return {"workload": f"{wl}, {args.solver}({args.m}) to {args.rtol:g}", "parallelism": f"replicas x{world}",
            "l2": "inputs > L2 (3.5 GB angular vector)"}


def workload_name(args):
    if args.mesh is None and args.groups is None:
        return True, "config1 multigroup dose solve: 768000 tets x 288 dirs x 20 groups, P5"
    n = tuple(args.mesh) if args.mesh else (40, 40, 80)
    NE = 6 * n[0] * n[1] * n[2]
    return False, f"reduced config1 physics (profiling case): {NE} tets x 288 dirs x {args.groups or 20} groups, P5"


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def rank_max(x):
    """Largest x over all ranks (replicas finish when the slowest one does); x itself on one rank.
    The reduction runs on the process group's device: the current GPU under NCCL, the host under gloo."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    dev = "cpu" if dist.get_backend() == "gloo" else f"cuda:{torch.cuda.current_device()}"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            parts = [p.strip() for p in l.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------------------------
#  CPU side: the FP64 oracle, a restatement of the reference's OpenMP CPU path (literal
#  encode / Sweep / decode for T^-1, the per-node dgemv loop of ScatteringAlgebra.f90:39-48 through
#  the OpenBLAS bundled with scipy for K), timed on the host cores.
# ---------------------------------------------------------------------------------------------
def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            return next(l.split(":", 1)[1].strip() for l in f if l.startswith("model name"))
    except (OSError, StopIteration):
        return "unknown"


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    return O


def cpu_operator_oracles(prob, threads, nd):
    """Oracles on the full mesh: one with nd evenly spaced directions and their sweep schedule (T^-1
    on complete directions), one with the full quadrature and no schedule (K)."""
    O = _oracle()
    O.set_threads(threads)
    O.set_blas()
    sigt, sigs = prob.within_group(0)
    sel = np.round(np.linspace(0, prob.NI - 1, nd)).astype(int)
    o_t = O.Oracle(prob.mesh)
    assert o_t.set_angular(prob.k[sel], prob.w[sel], prob.Ls, literal=False) == 0
    o_t.set_xs(sigt, sigs)
    o_k = O.Oracle(prob.mesh)
    assert o_k.set_angular_no_schedule(prob.k, prob.w, prob.Ls) == 0
    o_k.set_xs(sigt, sigs)
    return o_t, o_k, sel


def cpu_operator_time(o_t, o_k, q, x, sd1):
    """Wall seconds of T^-1 on q (o_t's directions) and of K on the nodes [0, sd1) of x."""
    t0 = time.perf_counter()
    o_t.transport_inv(q, inplace=True)
    t1 = time.perf_counter()
    o_k.scatter_apply_dgemv(x, 0, sd1, inplace=True)
    return t1 - t0, time.perf_counter() - t1


def fixture_iterations():
    """Operator applications per group of the FP64 moment-space oracle at 1e-6 on the benchmarked
    problem (tests/golden/config1_oracle.npz), or None."""
    path = os.path.join(ROOT, "tests", "golden", "config1_oracle.npz")
    if not os.path.exists(path):
        return None
    return np.load(path)["iters_snap"].astype(int)


def cpu_baseline(prob, threads):
    """One complete operator application of the FP64 CPU path on the benchmarked problem (T^-1 over
    all 288 directions, K on all 3,072,000 nodes), and a complete small-problem solve (6,000 tets, 80
    directions, GMRES(20) to 1e-8 in the reference's angular space)."""
    from lionbolt_b200 import problems as P
    O = _oracle()
    O.set_threads(threads)
    O.set_blas()
    t_setup = time.perf_counter()
    o_t = O.Oracle(prob.mesh)
    assert o_t.set_angular(prob.k, prob.w, prob.Ls, literal=False) == 0
    o_t.set_xs(*prob.within_group(0))
    n = prob.mesh.NENK * prob.NI
    x = np.random.default_rng(0).uniform(size=n)
    t_setup = time.perf_counter() - t_setup
    t_t, t_k = cpu_operator_time(o_t, o_t, x, x, prob.mesh.NENK)
    del x, o_t
    updates = prob.mesh.NE * prob.NI
    # complete small solve
    c0 = P.config0()
    o0 = O.Oracle(c0.mesh)
    o0.set_angular(c0.k, c0.w, c0.Ls, literal=False)
    o0.set_xs(c0.sigt[0], c0.sigs[0, 0])
    q0 = np.random.default_rng(1).uniform(size=c0.mesh.NENK * c0.NI)
    t0 = time.perf_counter()
    _, info = o0.boltzmann_solve(q0, "GMRES", m=20, rtol=1e-8, atol=0.0)
    t_c0 = time.perf_counter() - t0
    nmv = info["iters"] + 1
    its = fixture_iterations()
    derived = None
    if its is not None:
        ops = int(its.sum()) + prob.G            # + the right-hand-side sweep of every group
        derived = {"time_to_dose_s": ops * (t_t + t_k), "operator_applications": ops,
                   "note": "measured operator time x the FP64 oracle's operator count at 1e-6 (moment space); "
                           "the reference's angular GMRES cannot hold this problem (85 GB workspace)"}
    return {"value": updates / (t_t + t_k), "unit": UNIT, "cores": threads, "kind": "port",
            "sample": (f"one complete operator application of the FP64 oracle on the 768k-tet problem: T^-1 over all "
                       f"{prob.NI} directions (literal encode/sweep/decode, {t_t:.2f} s) + K through the per-node "
                       f"OpenBLAS dgemv path on all {prob.mesh.NENK} nodes ({t_k:.2f} s)"),
            "cpu": cpu_model(), "nproc": os.cpu_count(), "transport_inv_s": t_t, "scatter_s": t_k,
            "setup_s": t_setup, "derived_config1": derived,
            "config0_solve": {"seconds": t_c0, "operator_applications": nmv, "status": info["status"],
                              "updates_per_s": c0.mesh.NE * c0.NI * nmv / t_c0,
                              "workload": "6000 tets x 80 dirs x 1 group, P3, angular GMRES(20) to 1e-8"}}


def training_problem(args, k):
    """Training problem k of the learned preconditioner: the benchmarked geometry with other seeded
    cross sections and another slab position."""
    from lionbolt_b200 import problems as P
    n = tuple(args.mesh) if args.mesh else (40, 40, 80)
    depth = 0.5 * n[2]
    z0 = depth * (0.08 + 0.25 * k)
    return P.multigroup_box(n=n, size=(0.5 * n[0], 0.5 * n[1], depth), G=args.groups or 20, seed=1000 + k,
                            slab=(z0, z0 + 0.05 * depth), name=f"train{k}")


def learned_comparison(args, mg, device, barrier, gmres_ms, gmres_dose, gmres_iters, phase_ms):
    """Train the per-cell network on plain-solver data (untimed), decide per group on a held-out
    problem whether the learned FGMRES beats plain GMRES there (untimed), then time FGMRES with that
    gating on the benchmarked problem; the plain-GMRES dose checks its answer."""
    from lionbolt_b200 import MultigroupSolver
    t0 = time.perf_counter()
    tr = MultigroupSolver(device=device)
    tr.lp_init(seed=7)
    total = 0
    for k in range(args.lp_problems):
        tr.set_problem(training_problem(args, k))
        total = tr.lp_generate(samples_per_group=args.lp_samples, iters=8, seed=total + 1)
    t_gen = time.perf_counter() - t0
    loss = tr.lp_train(steps=args.lp_steps, batch=2048, lr=3e-3, seed=11)
    w = tr.lp_get_weights()
    t_train = time.perf_counter() - t0 - t_gen
    # held-out calibration: another seed and slab position than every training problem
    tr.set_problem(training_problem(args, args.lp_problems))
    plain_v, learned_v = tr.lp_calibrate(m=args.m, rtol=args.rtol)
    tr.Destroy()
    t_cal = time.perf_counter() - t0 - t_gen - t_train
    # a learned application costs one operator application plus the network (about a tenth of one)
    enabled = (1.1 * learned_v < plain_v).astype(np.int32)
    mg.lp_set_weights(w)
    mg.lp_set_groups(enabled, budget=plain_v)
    h = mg._h
    warm = min(args.warmup, 1)
    for _ in range(warm):
        mg.solve("FGMRES_ML", m=args.m, rtol=args.rtol, atol=0.0)
    barrier()
    h.mark(2)
    it = None
    for _ in range(args.steps):
        it = mg.solve("FGMRES_ML", m=args.m, rtol=args.rtol, atol=0.0)
    h.mark(3)
    ml_ms = rank_max(h.elapsed_ms(2, 3)) / args.steps
    _, dose = mg.results()
    mg.lp_enable(False)
    mg.lp_set_groups(None)
    rel = float(np.linalg.norm(dose - gmres_dose) / max(np.linalg.norm(gmres_dose), 1e-300))
    # Upper bound of any right preconditioner: an exact, free A^-1 makes FGMRES converge after the
    # initial-residual application and one more per group (plus the right-hand-side sweep); the time
    # of everything else is unchanged.  Per-application time from the plain solve's phase timers.
    G = len(gmres_iters)
    nmv = int(np.sum(gmres_iters))
    t_app = sum(phase_ms.get(k, 0.0) for k in ("sweep", "m2d", "d2m", "krylov")) / (nmv + G)
    t_other = gmres_ms - t_app * (nmv + G)
    bound = gmres_ms / (t_other + t_app * 3 * G)
    bound_zero_guess = gmres_ms / (t_other + t_app * 2 * G)
    return {"solver": f"FGMRES({args.m}) + per-cell MLP right preconditioner, gated per group",
            "time_to_dose_s": ml_ms / 1e3, "speedup_vs_gmres": gmres_ms / ml_ms,
            "iterations_per_group": [int(x) for x in it], "gmres_iterations_per_group": [int(x) for x in gmres_iters],
            "dose_rel_l2_vs_gmres": rel, "warmup": warm, "steps": args.steps,
            "gating": {"heldout_plain": plain_v.tolist(), "heldout_learned": learned_v.tolist(),
                       "enabled_groups": int(enabled.sum()), "rule": "learned x 1.1 < plain on a held-out problem",
                       "calibrate_s": t_cal},
            "bound_exact_inverse": {"speedup": bound, "speedup_zero_initial_guess": bound_zero_guess,
                                    "ms_per_application": t_app,
                                    "note": "free exact A^-1: 2 applications per group + the right-hand side"},
            "training": {"problems": args.lp_problems, "samples": int(total), "adam_steps": int(args.lp_steps),
                         "loss_first20": float(np.mean(loss[:20])), "loss_last50": float(np.mean(loss[-50:])),
                         "generate_s": t_gen, "train_s": t_train}}


def real_sh(Ls, dirs):
    """Real orthonormal spherical harmonics Y[i][l*l+l+m] (cos for m > 0, sin for m < 0), FP64."""
    dirs = np.asarray(dirs, dtype=np.float64)
    ct = dirs[:, 2]
    st = np.sqrt(np.maximum(0.0, 1.0 - ct * ct))
    ph = np.arctan2(dirs[:, 1], dirs[:, 0])
    Pl = {}
    Pl[(0, 0)] = np.ones_like(ct)
    for m in range(1, Ls + 1):
        Pl[(m, m)] = Pl[(m - 1, m - 1)] * (2 * m - 1) * st
    for m in range(Ls):
        Pl[(m + 1, m)] = (2 * m + 1) * ct * Pl[(m, m)]
    for m in range(Ls + 1):
        for l in range(m + 2, Ls + 1):
            Pl[(l, m)] = ((2 * l - 1) * ct * Pl[(l - 1, m)] - (l + m - 1) * Pl[(l - 2, m)]) / (l - m)
    Y = np.zeros((dirs.shape[0], (Ls + 1) ** 2))
    for l in range(Ls + 1):
        for m in range(-l, l + 1):
            am = abs(m)
            nrm = np.sqrt((2 * l + 1) / (4 * np.pi) * np.prod(1.0 / np.arange(l - am + 1, l + am + 1, dtype=np.float64)))
            v = nrm * Pl[(l, am)]
            if m > 0:
                v = v * np.sqrt(2.0) * np.cos(am * ph)
            elif m < 0:
                v = v * np.sqrt(2.0) * np.sin(am * ph)
            Y[:, l * l + l + m] = v
    return Y


# kernel of each sweep schedule the autotuner can pick
SWEEP_KERNELS = {"cluster levels": "sweep_cluster_kernel", "cluster levels+type tables": "sweep_cluster_kernel",
                 "cluster levels+element prefetch": "sweep_cluster_kernel",
                 "cluster levels+element prefetch+previous in registers": "sweep_cluster_kernel",
                 "cluster levels+element prefetch+two previous in registers": "sweep_cluster_kernel",
                 "cluster levels+type tables+element prefetch": "sweep_cluster_kernel",
                 "levels": "sweep_levels_kernel",
                 "levels+prefetch": "sweep_levels_pf_kernel", "element flags": "sweep_flags_kernel",
                 "grouped directions": "sweep_group_kernel", "dataflow": "sweep_dataflow_kernel"}


def run_gemm(args, steps=None, warmup=None, emit=True):
    """Standalone scattering contractions (config2 shapes): M2D psi[288][3,072,000] = Y[288][36]
    phi[36][3,072,000] and D2M phi = (wY)^T psi, on the device.  Split-BF16 tensor-core kernels vs
    cuBLAS FP32 (TF32 off) vs an FP64 reference on 65,536 sampled node columns."""
    import ctypes
    import torch
    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    from lionbolt_b200 import AngularClass, ScatteringOp, XSType
    from lionbolt_b200 import problems as P
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    prob = P.config1()
    m = prob.mesh
    NENK, NI, Ls = m.NENK, prob.NI, 5
    nm = (Ls + 1) ** 2
    op = ScatteringOp(device=local).Build(m, AngularClass(k=prob.k, w=prob.w),
                                          XSType(np.ones(m.Nm), np.ones((m.Nm, Ls + 1))))   # sigma_l = 1
    h = op._h
    dev = f"cuda:{local}"
    gen = torch.Generator(device=dev).manual_seed(20261203)
    lofj = np.concatenate([[l] * (2 * l + 1) for l in range(Ls + 1)])
    scale = torch.from_numpy(0.8 ** lofj).to(dev)
    phi = torch.randn(nm, NENK, dtype=torch.float64, device=dev, generator=gen) * scale[:, None]
    psi = torch.empty(NI, NENK, dtype=torch.float32, device=dev)
    phi2 = torch.empty(nm, NENK, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    vp = ctypes.c_void_p

    def timed(fn, slot):
        for _ in range(warmup):
            fn()
        h.call("lb_synchronize")
        h.mark(slot)
        for _ in range(steps):
            fn()
        h.mark(slot + 1)
        return h.elapsed_ms(slot, slot + 1) / steps

    t_m2d = timed(lambda: h.call("lb_m2d_device", vp(phi.data_ptr()), vp(psi.data_ptr())), 0)
    t_d2m = timed(lambda: h.call("lb_d2m_device", vp(psi.data_ptr()), vp(phi2.data_ptr())), 2)
    h.call("lb_synchronize")
    # cuBLAS FP32 comparators on the same inputs
    torch.backends.cuda.matmul.allow_tf32 = False
    Y = torch.from_numpy(real_sh(Ls, prob.k)).to(dev)                   # [NI, nm] FP64
    D = (Y * torch.from_numpy(prob.w).to(dev)[:, None]).T.contiguous()  # [nm, NI]
    Y32, D32, phi32 = Y.float(), D.float(), phi.float()

    def tevent(fn):
        for _ in range(warmup):
            fn()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record()
        for _ in range(steps):
            out = fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / steps, out

    t_m2d32, psi32 = tevent(lambda: Y32 @ phi32)
    t_d2m32, phi2_32 = tevent(lambda: D32 @ psi)
    # FP64 reference (CPU) on sampled columns; D2M uses the product's psi as input for every path
    cols = torch.randint(NENK, (65536,), generator=gen, device=dev)
    Yh, Dh = Y.cpu().numpy(), D.cpu().numpy()
    ref_m2d = Yh @ phi[:, cols].cpu().numpy()
    psi_s = psi[:, cols].double().cpu().numpy()
    ref_d2m = Dh @ psi_s
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    e_m2d = rel(psi[:, cols].double().cpu().numpy(), ref_m2d)
    e_m2d32 = rel(psi32[:, cols].double().cpu().numpy(), ref_m2d)
    e_d2m = rel(phi2[:, cols].cpu().numpy(), ref_d2m)
    e_d2m32 = rel(phi2_32[:, cols].double().cpu().numpy(), ref_d2m)
    flops = 2.0 * NENK * nm * NI
    by_m2d = NENK * (nm * 8 + NI * 4)
    by_d2m = NENK * (NI * 4 + nm * 8)
    peak, kind = measured_peaks()

    def entry(ms, by, err, ms32, err32):
        return {"ms": ms, "gbs": by / ms / 1e6, "hbm_frac": by / ms / 1e6 / peak, "useful_tflops": flops / ms / 1e9,
                "rel_l2_vs_fp64": err, "cublas_fp32": {"ms": ms32, "rel_l2_vs_fp64": err32}}

    line = {"metric": "config2 scattering contractions: split-BF16 (6 products, FP32 accumulate) vs FP32 vs FP64",
            "workload": f"M2D [{NI} x {nm}] x [{nm} x {NENK}] and D2M [{nm} x {NI}] x [{NI} x {NENK}], "
                        "phi ~ N(0,1) 0.8^l, seeded",
            "steps": steps, "warmup": warmup, "peak_gbs": peak, "peak_source": kind,
            "m2d": entry(t_m2d, by_m2d, e_m2d, t_m2d32, e_m2d32),
            "d2m": entry(t_d2m, by_d2m, e_d2m, t_d2m32, e_d2m32),
            "sample_columns": int(cols.numel()),
            "algorithmic_bytes": {"m2d": by_m2d, "d2m": by_d2m}}
    if rank == 0 and emit:
        print(json.dumps(line), flush=True)
    op.Destroy()
    del phi, psi, phi2, psi32, phi2_32, Y32, D32, phi32
    torch.cuda.empty_cache()
    return line


def run_batch(args, steps=None, warmup=None, emit=True):
    """Batched workload: 64 seeded independent dose problems solved together (one step = all 64)."""
    import torch
    from lionbolt_b200 import BatchSolver
    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    from lionbolt_b200 import problems as P
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    probs = P.batch_problems(count=args.batch_count, seed=20261203)
    bs = BatchSolver(device=local)
    for p in probs:
        bs.add_problem(p)
    for _ in range(warmup):
        bs.solve(m=args.m, rtol=args.rtol)
    torch.cuda.synchronize()
    ms, it = [], None
    with ClockSampler(local) as clocks:
        if args.profile_range:
            torch.cuda.profiler.start()
        for _ in range(steps):
            it = bs.solve(m=args.m, rtol=args.rtol)
            ms.append(bs.info()["last_ms"])
        if args.profile_range:
            torch.cuda.profiler.stop()
    info = bs.info()
    t = float(np.sum(ms))
    NE = np.array([p.mesh.NE for p in probs])
    NI = np.array([p.NI for p in probs])
    upd = float(sum(int(NE[i]) * int(NI[i]) * int(it[i].sum()) for i in range(len(probs))))
    nprob = len(probs)
    line = {"metric": f"batched dose solves (config3): {nprob} independent problems per step", "value": nprob * steps / (t / 1e3),
            "unit": "dose solves/s", "n_gpus": 1, "steps": steps, "warmup": warmup,
            "ms_per_step": t / steps, "higher_is_better": True, "dtype": "f32 sweep / split-bf16 moments / f64 Krylov",
            "data": "synthetic",
            "config": {"workload": f"{nprob} problems: hexes per axis U{{8..32}} x 6 tets, S8/S12/S16, 1-10 groups, P3, "
                                   f"GMRES({args.m}) to {args.rtol:g}, seed 20261203",
                       "tets_total": int(NE.sum()), "groups_total": int(sum(p.G for p in probs))},
            "updates_per_s": upd / (t / steps / 1e3),
            "operator_applications": int(it.sum()), "sweep_threads": info["sweep_threads"],
            "graph_launches": info["graph_launches"], "sweep_launches": info["sweep_launches"],
            "clocks": clocks.summary()}
    if rank == 0 and emit:
        print(json.dumps(line), flush=True)
    bs.close()
    return line


def general_mesh(spec):
    """A mesh for --workload mesh: a .npz fixture (rg, node, mat), a gmsh .msh file, or "jittered" (the
    40 x 40 x 80-hex box of the dose workload with every interior node moved by up to 0.15 of a hex
    edge, so that no two tets share a shape: 64-byte element records and the element-level sweep)."""
    from lionbolt_b200 import mesh as M
    if spec == "jittered":
        m = M.box_mesh(40, 40, 80, (0, 0, 0), (20.0, 20.0, 40.0),
                       material=lambda c: ((c[:, 2] >= 5.0) & (c[:, 2] <= 7.0)).astype(np.int32), Nm=2)
        rg = m.rg.copy()
        lo, hi = rg.min(axis=0), rg.max(axis=0)
        inner = np.all((rg > lo + 1e-9) & (rg < hi - 1e-9), axis=1)
        rg[inner] += 0.075 * np.random.default_rng(5).uniform(-1, 1, size=(int(inner.sum()), 3))
        return M.Mesh(rg=rg, node=m.node, neighbors=m.neighbors, mat=m.mat, Nm=2), "768000-tet box, jittered nodes"
    if spec.endswith(".npz"):
        d = np.load(spec)
        node = d["node"].astype(np.int32)
        mat = d["mat"].astype(np.int32)
        return (M.Mesh(rg=d["rg"], node=node, neighbors=M.neighbours(node), mat=mat, Nm=int(mat.max()) + 1),
                os.path.basename(spec))
    return M.read_gmsh(spec), os.path.basename(spec)


def run_mesh(args):
    """Sweep throughput of a within-group solve (288 directions, P5, c = 0.9, g = 0.95) on a general
    mesh; the sweep's algorithmic bytes (lb_sweep_stats) over its device time give the roofline."""
    import torch
    from lionbolt_b200 import AngularClass, BoltzmannOp, XSType
    from lionbolt_b200 import problems as P
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    m, name = general_mesh(args.mesh_file)
    k, w = P.quadrature(12, 24)
    sigt = np.array([0.2, 0.54])[:m.Nm]
    sigs = np.array([[0.9 * s * 0.95 ** l for l in range(6)] for s in sigt])
    L = BoltzmannOp(device=local, m=args.m, rtol=args.rtol, atol=0.0).Build(m, AngularClass(k=k, w=w),
                                                                         XSType(sigt, sigs))
    h = L._h
    q = np.random.default_rng(0).uniform(size=m.NENK * k.shape[0])
    # the first sweeps of a handle time the schedule candidates: warm up until the tuner has chosen
    for w in range(100):
        L.MatInv(q.copy())
        if w + 1 >= args.warmup and h.sweep_config() is not None:
            break
    h.reset_timers()
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            L.MatInv(q.copy())
    tm = h.timers()
    by, up, nz = np.zeros(1), np.zeros(1), np.zeros(1, dtype=np.int64)
    h.call("lb_sweep_stats", _lib_mod().dptr(by), _lib_mod().dptr(up), nz.ctypes.data_as(_lib_mod()._c_ll_p))
    sw_ms, sw_n = tm["sweep"]
    per = sw_ms / max(sw_n, 1)
    peak, kind = measured_peaks()
    gbs = by[0] / (per / 1e3) / 1e9
    launch = h.sweep_config() or {}
    line = {"metric": "sweep throughput on a general mesh", "mesh": name, "tets": m.NE, "element_types": h.mesh_types(),
            "directions": int(k.shape[0]), "sweep_ms": per, "sweeps": sw_n, "updates_per_s": up[0] / (per / 1e3),
            "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
                         "peak_source": kind, "algorithmic_bytes": float(by[0]),
                         "kernel": SWEEP_KERNELS.get(launch.get("schedule"), "sweep")},
            "launch": launch, "operator_applications": L.iters, "clocks": clocks.summary()}
    if rank == 0:
        print(json.dumps(line), flush=True)
    L.Destroy()
    return line


def _lib_mod():
    from lionbolt_b200 import _lib
    return _lib


REF_FRACTION = 4   # a reference step is 1/REF_FRACTION of one complete operator application


def run_reference(args):
    """The FP64 CPU path (the oracle, kind "port": the Fortran reference has no compiler here) on all host
    cores.  A step is a complete 1/4 of one operator application of the benchmarked problem: T^-1 over 72
    of the 288 directions on the full 768k-tet mesh and K through the per-node dgemv path on a quarter of
    the 3,072,000 nodes.  value = cell-direction-group updates of the step / its wall time."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from lionbolt_b200 import problems as P
    prob = P.config1()
    threads = os.cpu_count() or 1
    nd = prob.NI // REF_FRACTION
    o_t, o_k, sel = cpu_operator_oracles(prob, threads, nd)
    rng = np.random.default_rng(0)
    q = rng.uniform(size=prob.mesh.NENK * nd)
    x = rng.uniform(size=prob.mesh.NENK * prob.NI)
    sd1 = prob.mesh.NENK // REF_FRACTION
    for _ in range(args.warmup):
        cpu_operator_time(o_t, o_k, q, x, sd1)
    tt, tk = [], []
    for _ in range(args.steps):
        a, b = cpu_operator_time(o_t, o_k, q, x, sd1)
        tt.append(a)
        tk.append(b)
    sec = (sum(tt) + sum(tk)) / args.steps
    updates = prob.mesh.NE * nd
    value = updates / sec
    its = fixture_iterations()
    sample = (f"FP64 oracle (CPU restatement of the reference's OpenMP path): per step T^-1 over {nd} of {prob.NI} "
              f"directions on the full 768000-tet mesh (literal encode/sweep/decode) + K through the per-node "
              f"OpenBLAS dgemv path on {sd1} of {prob.mesh.NENK} nodes (1/{REF_FRACTION} of one operator "
              f"application); {NE_NI_NOTE}")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": bench_config(args, world),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
                             "cpu": cpu_model(), "nproc": os.cpu_count()},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "transport_inv_s_per_step": sum(tt) / args.steps, "scatter_s_per_step": sum(tk) / args.steps,
            "derived_time_to_dose_s": (None if its is None else
                                       (int(its.sum()) + prob.G) * sec * REF_FRACTION)}
    print(json.dumps(line), flush=True)
    return 0


def fixture_errors(prob, flux, dose):
    """Relative L2 errors of the dose and every group's fluence against the FP64 oracle's converged
    solution of the benchmarked problem (tests/golden/config1_oracle.npz): on the fixture's 4096
    sampled DG nodes, on the per-z-layer sums (every node), and of the full-vector norms."""
    path = os.path.join(ROOT, "tests", "golden", "config1_oracle.npz")
    if not os.path.exists(path):
        return None
    d = np.load(path)
    nodes = d["nodes"]
    nx, ny, nz = prob.mesh.shape
    layers = lambda v: v.reshape(nz, -1).sum(axis=1)
    rel = lambda a, b: float(np.linalg.norm(np.asarray(a) - b) / np.linalg.norm(b))
    fl = [rel(flux[g, nodes], d["flux"][g]) for g in range(prob.G)]
    return {"dose_rel_l2": rel(dose[nodes], d["dose"]), "flux_rel_l2_max": max(fl), "flux_rel_l2": fl,
            "dose_layers_rel_l2": rel(layers(dose), d["dose_layers"]),
            "flux_layers_rel_l2_max": max(rel(layers(flux[g]), d["flux_layers"][g]) for g in range(prob.G)),
            "dose_norm_rel": abs(float(np.linalg.norm(dose)) / float(d["dose_norm"]) - 1.0),
            "oracle": "FP64 moment-space GMRES(20) to 1e-10 (converged), tests/golden/config1_oracle.npz",
            "oracle_1e-6_dose_rel_l2": float(d["snap_dose_rel_l2"])}


def beam_subbench(prob, mg):
    """The first-collision data of the benchmarked beam ray-traced on the device (lb_beam_uncollided:
    4 quadrature points per element walked back to the beam plane, Beer's law, DG projection), with the
    beam plane 2 cm before the mesh; device time of the kernel from the phase timers."""
    b = np.asarray(prob.beam_dir, dtype=np.float64)
    e1 = np.cross([0.0, 1.0, 0.0], b)
    e1 /= np.linalg.norm(e1)
    e2 = np.cross(b, e1)
    sx, sy = prob.mesh.rg[:, 0].max(), prob.mesh.rg[:, 1].max()
    origin = np.array([0.5 * sx, 0.5 * sy, 0.0]) - 2.0 * b
    h = mg._h
    mg.beam_uncollided(origin, b, e1, e2, 5.0, 5.0, prob.sigt[0])          # device set-up on first use
    reps = 3
    t0 = h.timers()["tally"]
    for _ in range(reps):
        unc = mg.beam_uncollided(origin, b, e1, e2, 5.0, 5.0, prob.sigt[0])
    t1 = h.timers()["tally"]
    ms = (t1[0] - t0[0]) / reps
    rays = 4 * prob.mesh.NE
    return {"ms": ms, "rays": rays, "rays_per_s": rays / (ms / 1e3), "nonzero_nodes": int(np.count_nonzero(unc)),
            "workload": "planar 5 x 5 cm beam 15 degrees off axis, plane 2 cm before the 768000-tet mesh, "
                        "4 rays per element walked tet to tet in FP64"}


def run_ours(args):
    rank, world, local = dist_env()
    import torch
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from lionbolt_b200 import MultigroupSolver
    from lionbolt_b200 import _lib

    prob, wl = workload(args)
    mg = MultigroupSolver(device=local).set_problem(prob)
    h = mg._h

    def step():
        return mg.solve(args.solver, m=args.m, rtol=args.rtol, atol=0.0)

    for _ in range(args.warmup):
        step()

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        h.call("lb_synchronize")

    # ---- device-timed region ----
    barrier()
    h.reset_timers()
    iters = None
    with ClockSampler(local) as clocks:
        if args.profile_range:
            torch.cuda.profiler.start()
        h.mark(0)
        for _ in range(args.steps):
            iters = step()
        h.mark(1)
        dev_ms = h.elapsed_ms(0, 1)
        if args.profile_range:
            torch.cuda.profiler.stop()
    barrier()
    tm = h.timers()
    launches = int(sum(v[1] for v in tm.values()))
    ms_per_step = rank_max(dev_ms) / args.steps

    # sweep roofline
    by, up, nz = np.zeros(1), np.zeros(1), np.zeros(1, dtype=np.int64)
    h.call("lb_sweep_stats", _lib.dptr(by), _lib.dptr(up), nz.ctypes.data_as(_lib._c_ll_p))
    sw_ms, sw_n = tm["sweep"]
    sweeps_per_step = sw_n / args.steps
    updates_per_step = float(up[0]) * sweeps_per_step        # NE * NI per sweep (one group)
    value = world * updates_per_step / (ms_per_step / 1e3)
    per_sweep_ms = sw_ms / max(sw_n, 1)
    achieved = by[0] / (per_sweep_ms / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    launch = h.sweep_config() or {}
    kernel = SWEEP_KERNELS.get(launch.get("schedule"), "sweep")
    traffic = None
    tp = os.path.join(ROOT, "profiles", "sweep_dram_traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            d = json.load(f)
        # dram bytes of one captured sweep of the same kernel, scaled by the update count of this workload
        if d.get("kernel") == kernel:
            traffic = d["dram_bytes"] * (up[0] / d["updates"])

    # ---- end-to-end through the C ABI with pinned host buffers ----
    NENK, G = prob.mesh.NENK, prob.G
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).pin_memory()
    h_sigt, h_sigs, h_dd, h_unc, h_dir = (pin(prob.sigt), pin(prob.sigs), pin(prob.dd), pin(prob.unc),
                                          pin(prob.beam_dir))
    h_dose = torch.empty(NENK, dtype=torch.float64).pin_memory()
    dp = lambda t: _lib.ctypes.cast(t.data_ptr(), _lib._c_double_p)
    h2d = sum(int(t.numel()) * 8 for t in (h_sigt, h_sigs, h_dd, h_unc, h_dir))
    d2h = NENK * 8
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        h.call("lb_mg_update_inputs", dp(h_sigt), dp(h_sigs), dp(h_dd), dp(h_unc), dp(h_dir))
        step()
        h.call("lb_mg_get_results", None, dp(h_dose))
    e2e_s = rank_max(time.perf_counter() - t0)
    e2e_value = world * updates_per_step * args.steps / e2e_s
    gmres_dose = h_dose.numpy().copy()

    # accuracy against the FP64 oracle's converged solution of the same problem
    accuracy = None
    if rank == 0 and workload_name(args)[0] and args.solver == "GMRES":
        flux, dose = mg.results()
        accuracy = fixture_errors(prob, flux, dose)

    learned = None
    if not args.no_learned and args.solver == "GMRES":
        learned = learned_comparison(args, mg, local, barrier, ms_per_step, gmres_dose, iters,
                                     {k: v[0] / args.steps for k, v in tm.items()})

    sub = {}
    if not args.no_subbench and world == 1:
        sub["first_collision"] = beam_subbench(prob, mg)
        mg.Destroy()
        mg = None
        sub["gemm"] = run_gemm(args, steps=10, warmup=3, emit=False)
        sub["batch"] = run_batch(args, steps=2, warmup=1, emit=False)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(prob, os.cpu_count() or 1)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32 sweep / split-bf16 tensor-core moments / f64 Krylov",
                "data": "synthetic", "config": bench_config(args, world),
                "time_to_dose_s": ms_per_step / 1e3, "dose_solves_per_s": world / (ms_per_step / 1e3),
                "updates_per_step": updates_per_step, "sweeps_per_step": sweeps_per_step,
                "iterations_per_group": [int(x) for x in iters],
                "accuracy_vs_fp64_oracle": accuracy,
                "phase_ms_per_step": {k: v[0] / args.steps for k, v in tm.items()},
                "sweep": {"ms": per_sweep_ms, "gbs": achieved, "updates_per_s": up[0] / (per_sweep_ms / 1e3),
                          "algorithmic_bytes": float(by[0]), "upstream_faces": int(nz[0]), "launch": launch},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic, "kernel": kernel,
                             "peak_source": peak_kind},
                "gpu_launches": launches,
                "clocks": clocks.summary(),
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "time_to_dose_s": e2e_s / args.steps},
                "cpu_baseline": cpu,
                "learned_preconditioner": learned}
        line.update(sub)
        print(json.dumps(line), flush=True)
    if mg is not None:
        mg.Destroy()
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "gemm":
        run_gemm(args)
        return 0
    if args.workload == "batch":
        run_batch(args)
        return 0
    if args.workload == "mesh":
        run_mesh(args)
        return 0
    if args.workload == "beam":
        from lionbolt_b200 import MultigroupSolver
        prob, wl = workload(args)
        mg = MultigroupSolver().set_problem(prob)
        line = beam_subbench(prob, mg)
        line["mesh"] = wl
        print(json.dumps(line), flush=True)
        mg.Destroy()
        return 0
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
