/*
 * lionbolt_b200.h -- C ABI of the B200 (sm_100a) transport-solve library.
 *
 * Drop-in boundary for Lionbolt's within-group transport solve.  The reference exposes this path
 * as Fortran type-bound procedures re-exported by src/LionboltAPI.f90:1-12; every entry point
 * below names the reference procedure it replaces.  A Fortran caller binds them with iso_c_binding
 * interfaces (bind(C, name="lb_...")) whose arguments follow the C types below one for one.
 *
 * Conventions
 *   - Plain pointers and sizes only; all host arrays are C-contiguous, 0-based.
 *   - Angular vectors use the reference layout of SpaceAngleVector%v
 *     (src/operators/LinearOperatorClass.f90:30-41): v[i * NENK + 4 * e + k] for direction i,
 *     element e, local node k, NENK = 4 * NE (linear tetrahedra).
 *   - Moment vectors: m[j * NENK + 4 * e + k], j = l*l + l + m the real spherical-harmonic index.
 *   - Every call returns an LB_* status.  The reference terminates through stophere(msg) on the
 *     same conditions; lb_last_error() returns the message.
 *   - One handle = one CUDA device + one stream.  A handle is not safe for concurrent use from
 *     several host threads (the reference GMRES driver is not re-entrant either,
 *     src/solvers/SPARSKIT.f90:32, third_party/SPARSKIT/iters.f:1942).
 */
#ifndef LIONBOLT_B200_H
#define LIONBOLT_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lb_handle lb_handle;

enum lb_status {
    LB_OK = 0,
    LB_ERR_ARG = 1,      /* invalid argument / size                                           */
    LB_ERR_CUDA = 2,     /* CUDA runtime error                                                */
    LB_ERR_OOM = 3,      /* device allocation failed                                          */
    LB_ERR_CYCLE = 4,    /* sweep ordering stagnated: cyclic dependency (SweepOrder.f90:178)  */
    LB_ERR_TIMEOUT = 5,  /* a bounded device-side wait gave up (sweep dependency or tensor-core
                            contraction pipeline); the call's results are invalid             */
    LB_ERR_NOCONV = 6,   /* Krylov iteration limit reached (SPARSKIT.f90:159-162, ipar(1)=-1) */
    LB_ERR_NAN = 7,      /* residual norm is NaN (SPARSKIT.f90:123-124)                       */
    LB_ERR_STATE = 8,    /* operator not ready (TransportOperator.f90:87-88)                  */
    LB_ERR_BREAKDOWN = 9 /* Krylov breakdown (SPARSKIT.f90:166-169, ipar(1)=-3)               */
};

enum lb_solver {
    LB_SOLVER_SI = 0,          /* source iteration, src/solvers/SourceIteration.f90           */
    LB_SOLVER_GMRES = 1,       /* restarted GMRES(m), third_party/SPARSKIT/iters.f:1901        */
    LB_SOLVER_FGMRES_ML = 2,   /* FGMRES(m) with the learned right preconditioner             */
    LB_SOLVER_FGMRES = 3       /* FGMRES(m), iters.f:2511-2795, with the diagonal right
                                  preconditioner of lb_set_right_precond_diag (identity if unset) */
};

/* phase timers reported by lb_get_timers (milliseconds of device time, CUDA events) */
enum lb_timer { LB_T_SWEEP = 0, LB_T_M2D = 1, LB_T_D2M = 2, LB_T_KRYLOV = 3, LB_T_COPY = 4, LB_T_PRECOND = 5,
                LB_T_TALLY = 6, LB_NTIMERS = 7 };

int lb_version(void);
const char* lb_status_string(int status);

/* Create / destroy a handle on CUDA device `device`.  Replaces the construction and %Destroy of
 * TransportOp / ScatteringOp / BoltzmannOp (TransportOperator.f90:431-445,
 * ScatteringOperator.f90:279-289, BoltzmannOperator.f90:328-338). */
int lb_create(int device, lb_handle** out);
int lb_destroy(lb_handle* h);
/* Copies the last error message (NUL-terminated, truncated to len) into buf. */
int lb_last_error(const lb_handle* h, char* buf, int len);

/* Mesh: replaces MeshClass + mesh%PostProcess (src/geometry/PostProcess.f90:3-461) and the space
 * part of the operators, TransportOp%Space (TransportOperator.f90:172-255) and ScatteringOp%Space
 * (ScatteringOperator.f90:100-152).  Linear tetrahedra with gmsh local node order.
 *   rg[NN][3]          node coordinates
 *   node[NE][4]        0-based node ids, gmsh tetrahedron order, positively oriented
 *   neighbors[NE][4]   element across local face f (gmsh faces {0,1,2},{0,1,3},{0,2,3},{1,2,3}),
 *                      -1 on the boundary (gmshprocessing.py:32-42,258-288)
 *   mat[NE]            0-based material index < Nm (Nm <= 256)
 * Outward normals follow PostProcess.f90:45-102 bit for bit (sorted face nodes, centroid sign). */
int lb_set_mesh(lb_handle* h, int NE, int NN, const double* rg, const int* node, const int* neighbors,
                const int* mat, int Nm);

/* Angular quadrature: replaces AngularClass (src/angular/SNPrep.f90:39-86) as consumed by
 * TransportOp%SpaceAngle (TransportOperator.f90:257-388) -> BuildSpaceAngle (SweepOrder.f90,
 * SweepArrays.f90).  k[NI][3] unit directions, w[NI] weights (sum 4 pi).  Builds the per-direction
 * wavefront schedule on the host; returns LB_ERR_CYCLE when a level adds no element. */
int lb_set_quadrature(lb_handle* h, int NI, const double* k, const double* w);

/* Fills the GL x Chebyshev product quadrature of SNPrep.f90:39-76 (Ng polar, Nc azimuthal;
 * the reference uses Nc = 2 Ng).  k[Ng*Nc][3], w[Ng*Nc]. */
int lb_sn_quadrature(int Ng, int Nc, double* k, double* w);

/* Within-group cross sections: replaces TransportOp%Physics (TransportOperator.f90:390-429) and
 * ScatteringOp%Physics (ScatteringOperator.f90:215-277).  sigt[Nm] = XS%t, sigs[Nm][Ls+1] =
 * XS%s(0:Ls, m) (Legendre moments of the within-group scattering cross section). */
int lb_set_xs(lb_handle* h, int Ls, const double* sigt, const double* sigs);

/* Sweep schedule for bit-exact checks against SweepOrder.f90:105-207 / SweepArrays.f90:34-92.
 *   sl[NI][NE]        element visited at sweep position es of direction i (sl(es,i), 0-based)
 *   upmask[NI][NE]    bit f set when local face f of sl[i][es] is upstream (IsUpstream)
 *   nlevels[NI]       number of wavefront levels per direction
 *   level_start[NI][NE+1]  start position of each level (entries past nlevels[i] undefined)
 * Any pointer may be NULL. */
int lb_get_schedule(lb_handle* h, int* sl, unsigned char* upmask, int* nlevels, int* level_start);

/* T^{-1} in place: replaces TransportOp%MatInv ('SWEEP', TransportOperator.f90:72-151), i.e.
 * EncodeSweep + Sweep (TransportAlgebra.f90:29-246) + decode.  s[NI*NENK] enters as source,
 * leaves as solution (FP64 host buffer; the sweep runs in FP32 on the device). */
int lb_transport_inv(lb_handle* h, double* s);

/* T^{-1} in place on a caller-owned device vector, without allocating: psi is the FP32 angular
 * vector [NI][NENK] in device memory of the handle's GPU (same layout as lb_transport_inv), 16-byte
 * aligned (LB_ERR_ARG otherwise, before anything is launched).  No
 * counterpart in the reference: it exists for callers that cannot allocate device memory at solve
 * time (a host framework that owns the allocator, a Fortran runtime that only passes pre-allocated
 * device arrays, a loop that must not hit cudaMalloc's implicit synchronisation).  Its dependency
 * counters live in a fixed 1 MiB file-scope device array (at most 262,144 direction-level pairs;
 * larger schedules return LB_ERR_ARG) that every GPU loading the library keeps until exit.  The
 * first call on a device looks up the array's device address.  The call runs the dataflow sweep
 * schedule (not the autotuned one of lb_transport_inv) on the handle's stream and waits for it, so
 * it cannot be stream-captured; writes to psi queued on other streams must be finished first (an
 * event wait or a host synchronisation).  All calls on a device share the array: calls that
 * overlap on the GPU race. */
int lb_transport_inv_noalloc(lb_handle* h, float* psi);

/* The two halves of K on caller-owned device arrays of the handle's GPU, asynchronous on the
 * handle's stream (lb_synchronize waits):
 *   lb_m2d_device: psi[i][n] = sum_j Y_j(k_i) sigma_l(j)(mat(n)) phi[j][n]   (phi FP64 [nm][NENK],
 *                  psi FP32 [NI][NENK]; moment-to-discrete with the current cross sections)
 *   lb_d2m_device: phi[j][n] = sum_i w_i Y_j(k_i) psi[i][n]                  (discrete-to-moment)
 * Both are split-BF16 tensor-core contractions (six BF16 products per term, FP32 accumulation).
 * With sigma_l = 1 they are the plain GEMMs Y phi and (wY)^T psi of ScatteringAlgebra.f90:13-55.
 * A contraction whose bounded pipeline wait gave up is reported by the next lb_synchronize (or the
 * next synchronous call of the handle) as LB_ERR_TIMEOUT. */
int lb_m2d_device(lb_handle* h, const double* phi, float* psi);
int lb_d2m_device(lb_handle* h, const float* psi, double* phi);

/* K x in place: replaces ScatteringOp%MatVec (ScatteringOperator.f90:39-70 ->
 * ScatteringAlgebra.f90:13-55).  Evaluated as moment-to-discrete (discrete-to-moment (x)). */
int lb_scatter_apply(lb_handle* h, double* x);

/* x <- x - T^{-1} K x: replaces BoltzmannOp%MatVec with Tprecond (BoltzmannOperator.f90:59-104). */
int lb_boltzmann_matvec(lb_handle* h, double* x);

/* Right preconditioner of LB_SOLVER_FGMRES: z_j = d[j] v_j on moment row j (j = l*l + l + m),
 * nm = (Ls+1)^2 of the current cross sections (<= 64); nm = 0 or d = NULL restores the identity.
 * SPARSKIT fgmres takes any right preconditioner through reverse communication (ipar(1) = 5); this
 * fixed one exists so that the flexible driver can be checked step for step. */
int lb_set_right_precond_diag(lb_handle* h, int nm, const double* d);

/* L^{-1} s in place: replaces BoltzmannOp%MatInv (BoltzmannOperator.f90:106-151).  The Krylov
 * iteration runs in flux-moment space (n = nm*NENK) with the SPARSKIT stopping test
 * ||b - A phi|| <= rtol ||b|| + atol on the moment residual; maxit <= 0 means unlimited.
 * iters = number of operator applications, resid = final residual norm. */
int lb_boltzmann_solve(lb_handle* h, double* s, int solver, int m, double rtol, double atol, int maxit,
                       int* iters, double* resid);

/* Multigroup downscatter solve with dose tally: replaces the group loop of src/main/Main.f90:326-476
 * (PIEISource :544-747, OpL%MatInv :434, tapes, CalculateDeposition :750-824,
 * TallyDeposition.f90:19) with device-resident flux moments instead of disk tapes.
 *   sigt[G][Nm]; sigs[G][G][Nm][Ls+1] transfer g'->g Legendre moments (sigs[g][g] within-group);
 *   dd[G][Nm] dose cross sections (XS%DD); unc[NENK] uncollided scalar flux of the beam in group 0
 *   at every DG node; beam_dir[3] its direction (monodirectional first-collision source). */
int lb_mg_set_problem(lb_handle* h, int G, int Ls, const double* sigt, const double* sigs, const double* dd,
                      const double* unc, const double* beam_dir);
/* Replaces the per-solve inputs of a problem already set with the same sizes (no allocation):
 * cross sections, dose cross sections, uncollided flux and beam direction. */
int lb_mg_update_inputs(lb_handle* h, const double* sigt, const double* sigs, const double* dd, const double* unc,
                        const double* beam_dir);
/* Runs every group to the stopping test; iters[G] receives operator applications per group. */
int lb_mg_solve(lb_handle* h, int solver, int m, double rtol, double atol, int maxit, int* iters);
/* flux[G][NENK] scalar fluence (collided + uncollided), dose[NENK]; either may be NULL. */
int lb_mg_get_results(lb_handle* h, double* flux, double* dose);

/* Uncollided fluence of a planar beam with a rectangular field, at the DG nodes, computed on the device:
 * replaces ExternalBeam%RayTrace (RayTracing.f90:152-379), FluenceQuadrature (FluenceQuadrature.f90:16-32)
 * and the projection of FCSSource (FCSSource.f90:134-169).  The 4 quadrature points of every element
 * whose point lies in the field (InField.f90:47-63: |((x - origin) perpendicular to axis) . e1| <=
 * width1/2, the same for e2) are traced back to their projection on the beam plane (origin, e1, e2)
 * through the mesh; exp(-sum sigma_t * length) (attn[Nm]: total cross sections of the beam's group) is
 * projected onto the element's linear DG basis.  The result (unit fluence at the plane) becomes the
 * uncollided flux of the handle's multigroup problem (call after lb_mg_set_problem / lb_mg_update_inputs,
 * which overwrite it) and is copied to unc[NENK] when unc is not NULL.  origin, axis, e1, e2: [3],
 * axis, e1, e2 orthonormal. */
int lb_beam_uncollided(lb_handle* h, const double* origin, const double* axis, const double* e1, const double* e2,
                       double width1, double width2, const double* attn, double* unc);

/* Records CUDA event `slot` (0..15) on the handle's stream; lb_elapsed_ms returns the device time
 * between two recorded slots (synchronising on the later one). */
int lb_mark(lb_handle* h, int slot);
int lb_elapsed_ms(lb_handle* h, int slot_a, int slot_b, double* ms);

/* Device-time phase timers (ms) accumulated since the last reset, and kernel launch counts. */
int lb_get_timers(lb_handle* h, double* ms, long long* launches);
int lb_reset_timers(lb_handle* h);
/* Algorithmic traffic of one full sweep and its update count (NE*NI): 16 B source read + 16 B
 * solution write per update, 12 B per upstream face, and the element record (16 B with the type
 * table, 64 B without) once per sweep; schedule records are not counted. */
int lb_sweep_stats(lb_handle* h, double* bytes_per_sweep, double* updates_per_sweep, long long* upstream_faces);
/* Waits for the handle's stream; LB_ERR_TIMEOUT if a contraction queued since the last check timed out. */
int lb_synchronize(lb_handle* h);
/* Failure-path check (no counterpart in the reference): launches one thread that waits, with the
 * contraction kernels' bounded wait cut to `polls` polls, on a pipeline barrier that nothing arrives
 * at.  The wait gives up and raises the handle's timeout flag; the call returns what the following
 * synchronisation reports, LB_ERR_TIMEOUT (message in lb_last_error), and clears the flag, so the
 * handle stays usable. */
int lb_probe_pipeline_timeout(lb_handle* h, long long polls);
/* Sweep launch shape picked by the autotuner: cfg[0] schedule (0 levels, 1 dataflow, 2 levels with
 * next-level prefetch, 3 element flags, 4 grouped directions, 5 blocks of 6 elements swept as
 * units, 6 the same with per-type element tables), cfg[1] threads per CTA, cfg[2] directions per CTA
 * (minimum CTAs per SM for 5 and 6), cfg[3] updates in flight per thread.  Returns
 * LB_ERR_STATE while candidates are still being timed (the first sweeps of a handle). */
int lb_get_sweep_config(lb_handle* h, int* cfg);

/* Number of distinct (element shape, material) types of the mesh when it has at most 256 of them
 * (the sweep then reads 16-byte element records and a per-type table); 0 otherwise (64-byte
 * records).  No counterpart in the reference. */
int lb_mesh_types(lb_handle* h, int* ntypes);

/* SPARSKIT givens (third_party/SPARSKIT/iters.f:3225-3262) as the Krylov drivers apply it: the
 * rotation (c, s) taking (x, y) to (r, 0); x or y NaN gives c = 1, s = 0, r = 0.  Diagnostic. */
int lb_givens(double x, double y, double* c, double* s, double* r);

/* Block schedule of the sweep (schedules 5 and 6): blocks of up to 6 face-connected elements swept as
 * units over each direction's block-level graph.  Blocks are 6 consecutive element ids when those are
 * face-connected (a hex of a box mesh split into 6 tets); otherwise they are grown greedily from face
 * neighbours.  A direction whose block graph has a cycle sweeps the blocks on the cycle element by
 * element (one record per element), so every sweepable mesh has a block schedule and record counts
 * differ between directions.  Built by lb_set_quadrature.
 *   lb_cluster_info: *nblocks = number of blocks (0: no block schedule), *max_levels = largest
 *     block-level count of a direction.
 *   lb_cluster_layout: rec_base[NI + 1] = offset of each direction's records, blk_elem[nblocks][6]
 *     (optional) = block members (-1: empty), *max_records = largest record count of a direction.
 *   lb_get_cluster_schedule: rec[rec_base[NI]][4] records in execution order (x = block index; y, z, w =
 *     two 16-bit slots each in execution order: member position in the block (3 b, 7 = empty),
 *     upstream-face mask << 3, outflow-face mask << 7), starts[NI][max_records + 1] block-level
 *     starts (relative to rec_base[i]), nlevels[NI].
 * Diagnostics for tests; no counterpart in the reference. */
int lb_cluster_info(lb_handle* h, int* nblocks, int* max_levels);
int lb_cluster_layout(lb_handle* h, long long* rec_base, int* blk_elem, int* max_records);
int lb_get_cluster_schedule(lb_handle* h, int* rec, int* starts, int* nlevels);


/* ---- Learned right preconditioner (no counterpart in the reference) ------------------------------
 * A per-cell MLP (19 -> 64 -> 64 -> 16, ReLU, 6,480 parameters, BF16 weights and activations with
 * FP32 accumulation) used by LB_SOLVER_FGMRES_ML as the right preconditioner of FGMRES(m).  For a
 * moment vector v it reads, per cell, the 16 cell-averaged moments j < 16 scaled by their RMS s,
 * sigma_t*ell, sigma_s0*ell and sigma_s0/sigma_t (ell = 4V/S, the mean chord) and returns
 * z = v + s * net(x) on the cell's nodes for j < 16 (z = v for j >= 16).  Parameter layout (FP32):
 * W1[64][19], b1[64], W2[64][64], b2[64], W3[16][64], b3[16].  Without weights, or when disabled,
 * LB_SOLVER_FGMRES_ML runs plain GMRES; with weights the learned iterate is checked by its true
 * residual and finished with plain GMRES when it misses the tolerance. */
int lb_lp_nparams(void);
/* He-uniform initialisation from `seed` (output layer scaled by 0.1); enables the network. */
int lb_lp_init(lb_handle* h, unsigned long long seed);
int lb_lp_set_weights(lb_handle* h, const float* w);
int lb_lp_get_weights(lb_handle* h, float* w);
/* on = 0 makes LB_SOLVER_FGMRES_ML run plain GMRES while keeping the weights. */
int lb_lp_enable(lb_handle* h, int on);
/* y[n][16] = net(x[n][19]) on the device (tensor-core inference kernel). */
int lb_lp_forward(lb_handle* h, int n, const float* x, float* y);
/* z = preconditioner(v) for host moment vectors v, z [nm][NENK] with the current cross sections. */
int lb_lp_apply(lb_handle* h, const double* v, double* z);
/* Loss 1/(2n) sum_k w_k |net(x_k) - t_k|^2 over n samples (w = NULL: all weights 1) and its
 * gradient (FP32, parameter layout above). */
int lb_lp_loss_grad(lb_handle* h, int n, const float* x, const float* t, const float* w, double* loss, float* grad);
/* Training data from plain-solver runs of the multigroup problem set on the handle: per group a
 * GMRES reference solve (rtol 1e-10), then `iters` source iterations from the first-flight
 * moments; samples_per_group cells drawn (seeded) from the (residual, error) pairs of those
 * iterates are appended to the handle's device-resident training set. */
int lb_lp_generate(lb_handle* h, int samples_per_group, int iters, unsigned long long seed, long long* total);
int lb_lp_num_samples(lb_handle* h, long long* n);
/* x[n][19], t[n][16] and loss weights w[n] of the stored samples (any may be NULL).  A sample's
 * target is (ebar - rbar)/s for the cell-averaged residual rbar and error ebar, s the RMS of rbar
 * over the 16 moments; its weight is s^2 over the mean square of the residual field's moments. */
int lb_lp_get_samples(lb_handle* h, float* x, float* t, float* w);
int lb_lp_clear_samples(lb_handle* h);
/* Per-group use of the learned path in lb_mg_solve with LB_SOLVER_FGMRES_ML: enabled[g] = 0 runs
 * plain GMRES on group g; budget[g] > 0 (budget may be NULL) caps group g's learned FGMRES at that
 * many operator applications, after which plain GMRES finishes from the learned iterate (default
 * cap 4m).  G = 0 clears both (every group learned, cap 4m). */
int lb_lp_set_groups(lb_handle* h, int G, const int* enabled, const int* budget);
/* Operator applications per group of the learned FGMRES(m) and of plain GMRES(m) to rtol on the
 * handle's multigroup problem (each group from the first-flight moments, the plain answer feeding
 * the groups below): the data for lb_lp_set_groups, taken on a problem other than the one solved. */
int lb_lp_calibrate(lb_handle* h, int m, double rtol, int* plain_iters, int* learned_iters);
/* `steps` Adam steps (cosine-decayed learning rate from lr to lr/20) on batches of `batch` samples
 * drawn from the training set; loss_hist[steps] (optional) receives the batch losses. */
int lb_lp_train(lb_handle* h, int steps, int batch, double lr, unsigned long long seed, double* loss_hist);


/* ---- Batched dose solves (no counterpart in the reference, which runs one problem per process) ---
 * Many independent multigroup problems -- own mesh, quadrature, cross sections and beam each -- on
 * one GPU.  Groups and GMRES(m) steps advance in lock step over the problems; one persistent sweep
 * launch covers every (problem, direction) pair; the matrix-vector product of an Arnoldi step is
 * replayed from a CUDA graph; converged problems drop out through a device-side mask. */
typedef struct lb_batch lb_batch;
int lb_batch_create(int device, lb_batch** out);
int lb_batch_destroy(lb_batch* b);
int lb_batch_last_error(const lb_batch* b, char* buf, int len);
/* Adds a problem (arguments as lb_set_mesh + lb_set_quadrature + lb_mg_set_problem); *id = index. */
int lb_batch_add_problem(lb_batch* b, int NE, int NN, const double* rg, const int* node, const int* neighbors,
                         const int* mat, int Nm, int NI, const double* k, const double* w, int G, int Ls,
                         const double* sigt, const double* sigs, const double* dd, const double* unc,
                         const double* beam_dir, int* id);
/* GMRES(m) dose solve of every problem; iters[P][Gmax] (optional) receives operator applications
 * per problem and group (0 for groups a problem does not have).  Returns the first nonzero Krylov
 * status of any problem (all problems are still solved). */
int lb_batch_solve(lb_batch* b, int m, double rtol, double atol, int maxit, int* iters);
/* flux[G][NENK], dose[NENK] of problem id (either may be NULL). */
int lb_batch_get_results(lb_batch* b, int id, double* flux, double* dose);
/* Problem count, largest group count, device time of the last solve (ms), sweep threads picked by
 * the tuner, graph replays and batched sweep launches so far.  Any pointer may be NULL. */
int lb_batch_info(lb_batch* b, int* nproblems, int* max_groups, double* last_ms, int* sweep_threads,
                  long long* graph_launches, long long* sweep_launches);

#ifdef __cplusplus
}
#endif

#endif /* LIONBOLT_B200_H */
