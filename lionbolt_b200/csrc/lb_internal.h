// Internal state and kernel launchers of the B200 transport-solve library.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>
#include "../../include/lionbolt_b200.h"

namespace lb {

// elements per block of the cluster sweep schedule (a hex of a box mesh split into 6 tets)
constexpr int kClusterSize = 6;

// Packed schedule item (one per element-direction, in sweep order):
//   bits 0-23 element id, bits 24-27 upstream-face mask, bits 28-31 outflow-face mask.
constexpr int kElemBits = 24;
constexpr int kMaxElems = 1 << kElemBits;
// Packed neighbour word (one per element face):
//   bits 0-23 neighbour element (0xFFFFFF on the boundary), bits 24-29 three 2-bit local node
//   indices in the neighbour of this face's nodes (gmsh face order), bits 30-31 two bits of the
//   element's material id (face f holds bits 2f, 2f+1).
constexpr uint32_t kNoNeighbour = 0xFFFFFFu;

// Sweep chunk: up to 32 consecutive items of one (direction, level).
//   x = direction | (count-1) << 24, y = first sweep position, z = global level id,
//   w = size of the previous level of the same direction (0 for the first level).
struct SweepStatus {
    int work;        // next chunk to claim
    int abort;       // set on any timeout; every warp stops
    int err;         // LB_ERR_TIMEOUT when set
    int err_chunk;   // chunk (dataflow) or direction (element flags) whose wait gave up
    int err_elem;    // element that waited (element flags)
    int err_dep;     // upstream element it waited for
    int err_pos;     // chunk start in the padded order
    int err_bit;     // the awaited done bit as last read
    int dbg_next;    // chunks claimed so far in that direction (x32)
    int dbg_done;    // elements completed in that direction
    int dbg_exited;  // warps that left the claim loop
    int dbg_len;     // padded length of the direction
};

struct Timer {
    cudaEvent_t a, b;
    int kind;
};

struct DeviceBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

struct Handle {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    int sm_count = 0;

    // ---- mesh (host) ----
    int NE = 0, NN = 0, Nm = 0;
    long long NENK = 0;
    std::vector<double> rg;        // [NN][3]
    std::vector<int> node, nbr;    // [NE][4]
    std::vector<int> mat;          // [NE]
    std::vector<double> nrm;       // [NE][4][3] FP64 outward unit normals
    std::vector<double> svec;      // [NE][4][3] area*n/volume (FP64)
    std::vector<uint32_t> nbrpack; // [NE][4]
    bool mesh_ready = false;
    int mesh_version = 0;          // bumped by every lb_set_mesh

    // ---- angular ----
    int NI = 0, NIpad = 0;         // directions, and rounded up to a multiple of 16
    std::vector<double> k, w;      // [NI][3], [NI]
    std::vector<int> items;        // [NI][NE] packed sweep items
    std::vector<int> lvl_start;    // concatenated level starts per direction
    std::vector<int> lvl_base;     // [NI+1] offset of each direction's levels in lvl_start
    std::vector<int> nlev;         // [NI]
    long long nz_upstream = 0;
    int nchunks = 0;
    int total_levels = 0;
    bool angle_ready = false;

    // ---- physics ----
    int Ls = -1, nm = 0, nmpad = 0, ybuilt_NI = -1;
    std::vector<double> sigt, sigs;  // within group: [Nm], [Nm][Ls+1]
    bool phys_ready = false;
    int xs_version = 0;              // bumped by every lb_set_xs

    // ---- device buffers ----
    float4* d_geom = nullptr;      // [NE][4] (snx, sny, snz, nbrpack)
    // meshes with few distinct (element shape, material) types (voxel-based meshes): the face vectors
    // and material of every type in a table, and per element a 16-byte record: the four neighbour
    // words with the 8-bit type index in the bits that otherwise carry the material
    int4* d_rec = nullptr;         // [NE]
    float4* d_gtab = nullptr;      // [ngeom][3] (snx, sny, snz)
    int* d_tmat = nullptr;         // [ngeom] material of each type
    int ngeom = 0;                 // number of types; 0: no table (use d_geom)
    // cluster schedule: blocks of up to kClusterSize face-connected elements swept as units (0 blocks:
    // none).  Blocks are kClusterSize consecutive ids when those are face-connected (box meshes: one hex
    // each); otherwise they are grown greedily from face neighbours and listed in blk_elem.  A direction
    // sweeps "units": whole blocks, except blocks on a dependency cycle of that direction's block graph,
    // which are split into single elements, so the number of records differs between directions.
    int4* d_crec = nullptr;        // block records in block-level order, direction i's from crec_base[i]
    long long* d_crec_base = nullptr;   // [NI + 1]
    int* d_blk_elem = nullptr;     // [nclusters][kClusterSize] members (-1: empty); null for consecutive ids
    std::vector<long long> crec_base_h;
    std::vector<int> blk_elem_h;
    int max_cluster_records = 0;   // largest record count of a direction
    long long cluster_levels_total = 0;   // block levels summed over the directions
    int* d_cl_start = nullptr;     // block-level starts, per direction (ncl[i] + 1 entries)
    int* d_cl_base = nullptr;      // [NI] offset of direction i's starts in d_cl_start
    int* d_ncl = nullptr;          // [NI] block levels per direction
    int nclusters = 0;
    int max_cluster_levels = 0;
    std::vector<int> cl_start_h, cl_base_h, ncl_h;   // host copies of d_cl_start, d_cl_base, d_ncl
    std::vector<int4> crec_h;                        // the block records (host-only handles)
    int* d_mat = nullptr;          // [NE]
    int* d_items = nullptr;        // [NI][NE]
    int4* d_chunks = nullptr;      // [nchunks]
    int* d_pitems = nullptr;       // padded items: every level of every direction padded to 32 with -1
    long long* d_pbase = nullptr;  // [NI+1] start of each direction in d_pitems
    long long npitems = 0;
    // directions whose schedules are bit-identical (same order, same face masks) share a walk
    std::vector<int> dir_class;    // [NI] class representative (smallest direction id of the class)
    std::vector<int> class_members;  // directions sorted by class
    std::vector<int> class_start;    // [nclass+1]
    int* d_groups = nullptr;       // per-CTA groups for the grouped sweep, built per group size
    int groups_gmax = 0, ngroups = 0;
    int* d_lvl_start = nullptr;    // concatenated level starts (copy of lvl_start)
    int* d_lvl_base = nullptr;     // [NI+1]
    int* d_nlev = nullptr;         // [NI]
    int* d_done = nullptr;         // [total_levels]
    SweepStatus* d_status = nullptr;
    int* d_tc_err = nullptr;      // set to LB_ERR_TIMEOUT by a contraction kernel whose pipeline wait gave up
    float4* d_dirs = nullptr;      // [NI] (kx, ky, kz, w)
    float* d_sigt = nullptr;       // [Nm]
    float* d_psi = nullptr;        // [NI][NENK] FP32 angular work vector
    float* d_qext = nullptr;       // [NI][NENK] FP32 angular external source (angular API)
    // moment-space operators (split BF16 hi/mid/lo planes)
    __nv_bfloat16* d_Ym2d = nullptr;  // [3][NIpad][nmpad] Y_j(k_i)
    __nv_bfloat16* d_Yd2m = nullptr;  // [3][nmpad][NIpad] w_i Y_j(k_i)
    float* d_sigl = nullptr;          // [Nm][nmpad]  sigma_l(j) per material (within group)
    int* d_lofj = nullptr;
    size_t psi_elems = 0;

    // ---- Krylov workspace (FP64, moment space) ----
    int kry_m = 0;
    double* d_V = nullptr;         // [(m+1)][N] basis
    double* d_Z = nullptr;         // [m][N] flexible basis (FGMRES)
    std::vector<double> pdiag;     // per-moment right-preconditioner scaling of LB_SOLVER_FGMRES (empty: identity)
    double* d_x = nullptr;         // solution
    double* d_b = nullptr;         // rhs
    double* d_t = nullptr;         // scratch
    double* d_red = nullptr;       // reduction partials
    double* h_red = nullptr;       // pinned host copy of reductions
    size_t kry_n = 0;

    // ---- multigroup ----
    int G = 0;
    std::vector<double> mg_sigt, mg_sigs, mg_dd;  // [G][Nm], [G][G][Nm][Ls+1], [G][Nm]
    std::vector<double> beam_dir;
    double* d_unc = nullptr;        // [NENK]
    double* d_phi_all = nullptr;    // [G][nm][NENK] collided flux moments
    double* d_src = nullptr;        // [nm][NENK] group source moments
    double* d_dose = nullptr;       // [NENK]
    double* d_flux = nullptr;       // [G][NENK]
    float* d_sigl_mg = nullptr;     // [G][G][Nm][nmpad] transfer tables sigma_l(j)
    double* d_yb = nullptr;         // [nm] beam-direction harmonics
    double* d_dd = nullptr;         // [G][Nm] dose cross sections
    int mg_alloc_G = 0, mg_alloc_nm = 0;
    long long mg_alloc_NENK = 0;
    size_t mg_alloc_tab = 0;

    // ---- timers ----
    std::vector<Timer> timers;
    std::vector<Timer> free_timers;
    double acc_ms[LB_NTIMERS] = {0};
    long long launches[LB_NTIMERS] = {0};

    // sweep launch configuration chosen by the online autotuner (sweep.cu)
    int sweep_cfg = -1;            // index into the candidate table, -1 = still tuning
    int sweep_trial = 0;
    std::vector<float> sweep_trial_ms;
    std::vector<int> sweep_finalists;   // candidates of the second timing round
    int sweep_cfg_forced = -1;     // set through LB_SWEEP_CONFIG for experiments

    cudaEvent_t marks[16] = {};

    // planar-beam ray walk (beam.cu): face planes, coordinates, connectivity, neighbours on the device
    double4* d_beam_plane = nullptr;
    double* d_beam_xyz = nullptr;
    int* d_beam_node = nullptr;
    int* d_beam_nbr = nullptr;
    int beam_mesh_version = -1;
    // learned preconditioner state (mlp.cu)
    void* mlp = nullptr;
    // per-group use of the learned path in multigroup solves (empty: every group) and the operator
    // applications after which a group's learned FGMRES gives way to plain GMRES (0: 4m)
    std::vector<char> lp_groups;
    std::vector<int> lp_budget;

    // batched solves (batch.cpp): a problem of a batch records no CUDA events (its launches may be
    // captured into graphs) and its moment kernels skip their work while *d_active == 0
    bool timing = true;
    const int* d_active = nullptr;
    // staging of segment tables for the segmented vector operations (krylov.cu)
    void* d_seg = nullptr;
    void* h_seg = nullptr;
    size_t seg_bytes = 0;
};

// ---- host helpers (host.cpp) ----
int fail(Handle* h, int code, const std::string& msg);
int cuda_fail(Handle* h, cudaError_t e, const char* what);
void real_sh(int Ls, const double* dir, double* Y);

// ---- learned preconditioner (mlp.cu) ----
void mlp_destroy(Handle* h);
bool mlp_ready(Handle* h);
// z = preconditioner(v); v * vscale is the vector the network's features are taken from (z in v's units)
int mlp_apply_precond(Handle* h, const double* v, double* z, double vscale);
// Appends `count` training samples drawn from the residual r and error err (device moment vectors).
int mlp_sample(Handle* h, const double* r, const double* err, long long count, unsigned long long seed);

// A value computed once per device at one call site (kernel attributes and occupancies are per
// device, and one process may drive several GPUs from several threads); the caller keeps it as a
// function-local static.
struct PerDevice {
    std::mutex m;
    unsigned long long done = 0;
    int value[64] = {};
    template <class F>
    int get(F&& f) {
        int dev = 0;
        cudaGetDevice(&dev);
        dev &= 63;
        std::lock_guard<std::mutex> g(m);
        if (!(done >> dev & 1ull)) {
            value[dev] = f();
            done |= 1ull << dev;
        }
        return value[dev];
    }
};

// Allow a kernel the largest dynamic shared memory the device permits next to its static
// shared memory (227 KB per CTA on sm_100 in total).  Clears the error state it may leave.
template <class K>
inline void allow_max_dynamic_smem(K kernel) {
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, kernel) != cudaSuccess) { cudaGetLastError(); return; }
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    int dyn = optin - (int)fa.sharedSizeBytes;
    if (dyn > 0) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
    cudaGetLastError();
}

// Krylov workspace of a handle for restart length m (solve.cpp)
int ensure_krylov(Handle* h, int m, bool flexible);
// multigroup helpers (solve.cpp): transfer table sigma_l(j) of g' -> g, beam harmonics, and the
// group source + within-group cross sections of group g (from the solved groups below it)
float* mg_table(Handle* h, int gp, int g);
void mg_prepare(Handle* h);
int mg_group_sources(Handle* h, int g);

// ---- batched solves ----
// One work item of the batched sweep: one direction of one problem of a batch.
struct BatchWork {
    const int* items;       // [NE] packed schedule items of the direction
    const int* lvl_start;   // [nlev + 1] level starts of the direction
    const float4* geom;     // the problem's element records
    const float* sigt;      // the problem's per-material total cross sections (device, FP32)
    float* psi;             // the problem's angular vector, block of this direction
    float4 dir;             // (kx, ky, kz, w)
    int nlev;
    int Nm;
    int problem;
    int ngeom;              // element types of the problem (0: no type table)
    const int4* crec;       // the direction's block records (nullptr: element schedule)
    const int* blk_elem;    // the problem's block members (nullptr: blocks of consecutive ids)
    const int* cl_start;    // [ncl + 1] block-level starts of the direction
    const int4* rec;        // the problem's 16-byte element records (type table)
    const float4* gtab;     // [ngeom][3] face vectors of the types
    const int* tmat;        // [ngeom] material of the types
    int ncl;
    int pad[3];
};
// Sweeps every work item whose problem has active[problem] != 0, CTAs claiming items in order from
// *counter (reset before the launch).  threads: 1024 or 512.
int launch_sweep_batch(cudaStream_t s, const BatchWork* work, int nwork, int* counter, const int* active,
                       int threads, int sm_count);

// Segmented (per-problem) FP64 vector operations of a batch: one launch for all problems.
struct SegVec {
    double* w;              // target vector (updated / dotted)
    const double* V;        // nv basis vectors, stride ldv
    const double* x;        // second operand of axpby
    double* w2;             // optional second destination of axpy_scale
    size_t ldv;
    size_t n2;              // vector length / 2
    int blk0, nblk;         // blocks of the launch assigned to this problem
    int coef;               // offset of this problem's coefficients
    int pad;
    double scale, a, b;
};
// Builds block ranges proportional to the vector lengths for a grid of `blocks`.
int seg_assign_blocks(std::vector<SegVec>& segs, int blocks);
// out[s][j] = V_j . w (j < nv) and out[s][nv] = w . w, for every segment s
int seg_dots_norm(Handle* h, const std::vector<SegVec>& segs, int nv, std::vector<double>& out);
// w -= sum_j c[s][j] V_j; out[s][j] = V_j . w (if dots) and out[s][nv] = w . w
int seg_axpy_dots(Handle* h, const std::vector<SegVec>& segs, int nv, const std::vector<double>& coef, bool dots,
                  std::vector<double>& out);
// w = (w - sum_j c[s][j] V_j) * scale (also written to w2 when non-null)
int seg_axpy_scale(Handle* h, const std::vector<SegVec>& segs, int nv, const std::vector<double>& coef);
// w = a x + b w and out[s] = w . w
int seg_axpby_norm(Handle* h, const std::vector<SegVec>& segs, std::vector<double>& out);

// ---- timers ----
void timer_begin(Handle* h, int kind, Timer& t);
void timer_end(Handle* h, Timer& t);
void timers_flush(Handle* h);

// ---- kernels (sweep.cu / moments.cu / krylov.cu) ----
// Full transport sweep psi <- T^{-1} psi (FP32, in place, natural layout [NI][NENK]).
int launch_sweep(Handle* h, float* psi);
// Chosen sweep launch shape (-1 while the autotuner is still timing candidates).
int sweep_config(Handle* h, int* kind, int* threads, int* dpc, int* ilp);
// q[i][n] = sum_j Y_j(k_i) * (sigl[mat(n)][j] * x[j][n] + a[j][n]) (+ qadd[i][n] if given).
// x and a are FP64 moment vectors [nm][NENK]; either may be null.
int launch_m2d(Handle* h, const double* x, const float* sigl, const double* a, const float* qadd, float* q);
// z[j][n] = sum_i w_i Y_j(k_i) psi[i][n]; out[j][n] = alpha * xin[j][n] + beta * z[j][n]
// (xin may be null: out = beta * z).
int launch_d2m(Handle* h, const float* psi, const double* xin, double alpha, double beta, double* out);

// tcgen05 versions of the two contractions (moments_tc.cu); LB_ERR_ARG when a shape does not fit them.
// LB_MOMENTS_TC=0 selects the mma.sync kernels.
bool moments_tc_enabled();
int launch_m2d_tc(Handle* h, const double* x, const float* sigl, const double* a, const float* qadd, float* q);
int launch_d2m_tc(Handle* h, const float* psi, const double* xin, double alpha, double beta, double* out);
// Reads and clears the tensor-core kernels' bounded-wait timeout flag.
int moments_tc_status(Handle* h);
// Runs the bounded pipeline wait against a barrier nothing arrives at (polls polls); returns what
// moments_tc_status reports afterwards.
int tc_wait_probe(Handle* h, long long polls);

// FP64 BLAS-1 on device vectors of length n
int k_dots(Handle* h, const double* V, size_t ldv, int nv, const double* w, size_t n, double* out_host);
// out[j] = V_j . w (j < nv, nv may be 0) and *wnorm2 = w . w in one pass (outputs may be null)
// zm: w holds z and the vector dotted is V_{nv-1} - z (k_axpy_dots: updated and written back to w).
int k_dots_norm(Handle* h, const double* V, size_t ldv, int nv, const double* w, size_t n, double* out, double* wnorm2,
                bool zm = false);
// w -= sum_j coef[j] V_j, then dots[j] = V_j . w and *nrm2 = w . w in the same pass (outputs may be null)
int k_axpy_dots(Handle* h, double* w, const double* V, size_t ldv, int nv, const double* coef, size_t n, double* dots,
                double* nrm2, bool zm = false);
// w <- (w - sum_j coef[j] V_j) * scale
int k_axpy_scale(Handle* h, double* w, const double* V, size_t ldv, int nv, const double* coef, double scale, size_t n);
int k_multi_axpy_norm(Handle* h, double* w, const double* V, size_t ldv, int nv, const double* coef, size_t n, double* nrm2);
// y <- a x + b y and *nrm2 = y . y
int k_axpby_norm(Handle* h, double* y, const double* x, double a, double b, size_t n, double* nrm2);
int k_multi_axpy(Handle* h, double* w, const double* V, size_t ldv, int nv, const double* coef_host, size_t n);
int k_axpby(Handle* h, double* y, const double* x, double a, double b, size_t n);   // y = a*x + b*y
int k_scale(Handle* h, double* y, double a, size_t n);
constexpr int kMaxRowCoefs = 64;   // moment rows of k_scale_rows (P7)
int k_scale_rows(Handle* h, double* z, const double* v, const double* coef, int nm, size_t NENK);   // z_j = c_j v_j
int k_copy(Handle* h, double* y, const double* x, size_t n);
int k_fill(Handle* h, double* y, double v, size_t n);
int k_f64_to_f32(Handle* h, float* y, const double* x, size_t n);
int k_f32_to_f64(Handle* h, double* y, const float* x, size_t n);
int k_dose_tally(Handle* h, const double* phi00, const double* unc, double unc_scale, const double* dd_mat,
                 const int* mat, double* flux, double* dose, long long NENK);
int k_moment_source(Handle* h, double* src, const double* phi, const float* sigl, const int* mat, long long NENK,
                    int nm, int nmpad, int accumulate);
// src = sum_{g'<g} Sigma_{g'->g} phi_{g'} + Sigma_{0->g} Y(beam) unc, one pass (tab: [G][G][Nm][nmpad])
int k_group_source(Handle* h, double* src, const double* phi_all, const float* tab, int G, int g, const double* unc,
                   const double* ybeam, const int* mat, long long NENK, int Nm, int nm, int nmpad);
int k_unc_source(Handle* h, double* src, const double* unc, const double* ybeam, const float* sigl, const int* mat,
                 long long NENK, int nm, int nmpad);

}  // namespace lb
