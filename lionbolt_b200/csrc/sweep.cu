// Discontinuous-Galerkin upwind sweep for linear tetrahedra, FP32, sm_100a.
//
// Replaces TransportAlgebra.f90:29-246 (Sweep + ApplyInvertedDiagonal + LocalLU) and the
// EncodeSweep.f90 permutations around it: the kernels index the natural-order vector through the
// per-direction schedule, so the encode/decode copies disappear.
//
// Element operator.  For linear tets the mass-eliminated matrices of
// FiniteElementAnalysis.f90:228-304 have closed forms in terms of the scaled face vectors
// s_f = A_f n_f / V (area, outward unit normal, volume).  With c_f = k . s_f:
//   -sum_d k_d IC_d (k,kp) = (5/3) c_{3-k}                  (face 3-k is opposite vertex k)
//   (k.n_f) IFM_f (k,kp) = c_f P_f(k,kp),   P_f(k,kp) = [kp in f] * (k==kp ? 2 : k in f ? 1/3 : -4/3)
//   (k.n_f) IIM_f = c_f P_f with columns mapped to the neighbour's local nodes.
// The 4x4 system  T = sigma I - sum_d k_d IC_d + sum_{f: k.n_f >= 0} (k.n_f) IFM_f  and the upstream
// coupling  rhs -= sum_{f upstream} (k.n_f) IIM_f psi_up  are therefore assembled from 12 floats
// per element.  T is a rank-2 update of a multiple of the identity, so the reference's pivoted LU
// (LocalLU) becomes a 2x2 capacitance solve with the same FP32 accuracy.
//
// Two schedules share that element update:
//  * levels (default): one CTA owns whole directions and walks their wavefront levels in order
//    with a CTA barrier between levels.  No global synchronisation; upstream values written by the
//    same SM are re-read through its L1.
//  * dataflow: warps claim 32-element chunks of (direction, level) in level-major order from a
//    global counter and wait, with a bounded spin, on the completion counter of the previous level.
// Launch shape (schedule, threads per CTA, directions per CTA, updates in flight per thread) is
// picked by timing the first sweeps of a handle; every candidate computes bit-identical results.
#include "lb_internal.h"
#include <cstdio>
#include <cstdlib>

namespace lb {

namespace {

constexpr float kThird = 1.0f / 3.0f;
constexpr float kFiveThirds = 5.0f / 3.0f;
constexpr float kFourThirds = 4.0f / 3.0f;

struct SweepArgs {
    const int* __restrict__ items;
    const int4* __restrict__ chunks;
    const int* __restrict__ lvl_start;
    const int* __restrict__ lvl_base;
    const int* __restrict__ nlev;
    int* done;
    const float4* __restrict__ geom;
    const float4* __restrict__ dirs;
    const float* __restrict__ sigt;
    float* psi;
    long long NENK;
    int NE;
    int NI;
    int nchunks;
    int Nm;
    SweepStatus* status;
    long long spin_limit;
};

__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ float pick(const float4& v, int idx) {
    float r = v.x;
    r = (idx == 1) ? v.y : r;
    r = (idx == 2) ? v.z : r;
    r = (idx == 3) ? v.w : r;
    return r;
}

// Loads of one element-direction update.  kCG selects L2-only loads (data written by other SMs).
template <bool kCG>
__device__ __forceinline__ float4 ld4(const float* p) {
    if (kCG) return __ldcg(reinterpret_cast<const float4*>(p));
    return *reinterpret_cast<const float4*>(p);
}

struct Update {
    float r[4];        // right-hand side, then solution
    float a[4], b[4];  // T = d I + a 1^T + 1 b^T
    float d;
};

// Assemble the element system of element e in direction dir.
//
// With c_f = k . s_f, co_f = c_f on outflow faces (k.n_f >= 0) else 0, ci_f = c_f - co_f and
// Ct = sum_f co_f, the matrix sigma I - sum_d k_d IC_d + sum_out (k.n_f) IFM_f equals
//   T = d I + a 1^T + 1 b^T,  d = sigma + (5/3) Ct,  a_k = (5/3) ci_{3-k},  b_k = (Ct - co_{3-k}) / 3
// (row k of the convection term is constant, column kp of the outflow term is constant off the
// diagonal), so the 4x4 solve reduces to a 2x2 one (Sherman-Morrison-Woodbury).
template <bool kCG>
__device__ __forceinline__ void assemble(const SweepArgs& a, const float* base, float4 dir, int item,
                                         const float* s_sigt, Update& u) {
    // gmsh face -> local nodes; the vertex opposite face f is 3 - f
    constexpr int F[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
    const int e = item & 0xFFFFFF;
    const int upm = (item >> 24) & 0xF;
    const int outm = (item >> 28) & 0xF;
    const float4 gx = __ldg(&a.geom[(size_t)e * 4 + 0]);
    const float4 gy = __ldg(&a.geom[(size_t)e * 4 + 1]);
    const float4 gz = __ldg(&a.geom[(size_t)e * 4 + 2]);
    const int4 gn = __ldg(reinterpret_cast<const int4*>(&a.geom[(size_t)e * 4 + 3]));
    const float4 q = ld4<kCG>(base + 4 * (size_t)e);
    float c[4];
    c[0] = fmaf(dir.x, gx.x, fmaf(dir.y, gy.x, dir.z * gz.x));
    c[1] = fmaf(dir.x, gx.y, fmaf(dir.y, gy.y, dir.z * gz.y));
    c[2] = fmaf(dir.x, gx.z, fmaf(dir.y, gy.z, dir.z * gz.z));
    c[3] = fmaf(dir.x, gx.w, fmaf(dir.y, gy.w, dir.z * gz.w));
    const unsigned nw[4] = {(unsigned)gn.x, (unsigned)gn.y, (unsigned)gn.z, (unsigned)gn.w};
    const int matid = (int)((nw[0] >> 30) | ((nw[1] >> 30) << 2) | ((nw[2] >> 30) << 4) | ((nw[3] >> 30) << 6));
    const float sig = s_sigt[matid];
    u.r[0] = q.x; u.r[1] = q.y; u.r[2] = q.z; u.r[3] = q.w;
    // upstream coupling: r -= (k.n_f) IIM_f psi_up over the inflow faces
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        if ((upm >> f) & 1) {
            const unsigned wd = nw[f];
            const int ep = (int)(wd & 0xFFFFFFu);
            const float4 u4 = ld4<kCG>(base + 4 * (size_t)ep);
            const float u0 = pick(u4, (wd >> 24) & 3);
            const float u1 = pick(u4, (wd >> 26) & 3);
            const float u2 = pick(u4, (wd >> 28) & 3);
            const float U = u0 + u1 + u2;
            const float cf = c[f];
            const float t3 = U * kThird;
            u.r[F[f][0]] = fmaf(-cf, fmaf(kFiveThirds, u0, t3), u.r[F[f][0]]);
            u.r[F[f][1]] = fmaf(-cf, fmaf(kFiveThirds, u1, t3), u.r[F[f][1]]);
            u.r[F[f][2]] = fmaf(-cf, fmaf(kFiveThirds, u2, t3), u.r[F[f][2]]);
            u.r[3 - f] = fmaf(cf * kFourThirds, U, u.r[3 - f]);
        }
    }
    float co[4];
#pragma unroll
    for (int f = 0; f < 4; ++f) co[f] = ((outm >> f) & 1) ? c[f] : 0.0f;
    const float Ct = (co[0] + co[1]) + (co[2] + co[3]);
    u.d = fmaf(kFiveThirds, Ct, sig);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        u.a[k] = kFiveThirds * (c[3 - k] - co[3 - k]);
        u.b[k] = (Ct - co[3 - k]) * kThird;
    }
}

// Solve (d I + a 1^T + 1 b^T) x = r through the 2x2 capacitance system
//   [d + sum a, 4; b.a, d + sum b] z = [sum r; b.r],   x = (r - a z0 - z1) / d.
__device__ __forceinline__ void solve_rank2(Update& u) {
    const float sa = (u.a[0] + u.a[1]) + (u.a[2] + u.a[3]);
    const float sb = (u.b[0] + u.b[1]) + (u.b[2] + u.b[3]);
    const float ba = fmaf(u.b[0], u.a[0], fmaf(u.b[1], u.a[1], fmaf(u.b[2], u.a[2], u.b[3] * u.a[3])));
    const float v0 = (u.r[0] + u.r[1]) + (u.r[2] + u.r[3]);
    const float v1 = fmaf(u.b[0], u.r[0], fmaf(u.b[1], u.r[1], fmaf(u.b[2], u.r[2], u.b[3] * u.r[3])));
    const float e00 = u.d + sa, e11 = u.d + sb;
    const float det = fmaf(e00, e11, -4.0f * ba);
    const float idet = __frcp_rn(det);
    const float z0 = fmaf(e11, v0, -4.0f * v1) * idet;
    const float z1 = fmaf(e00, v1, -ba * v0) * idet;
    const float id = __frcp_rn(u.d);
#pragma unroll
    for (int k = 0; k < 4; ++k) u.r[k] = (u.r[k] - fmaf(u.a[k], z0, z1)) * id;
}

template <bool kCG>
__device__ __forceinline__ void finish(float* base, int item, Update& u) {
    solve_rank2(u);
    const int e = item & 0xFFFFFF;
    float4 v = make_float4(u.r[0], u.r[1], u.r[2], u.r[3]);
    if (kCG) __stcg(reinterpret_cast<float4*>(base + 4 * (size_t)e), v);
    else *reinterpret_cast<float4*>(base + 4 * (size_t)e) = v;
}

__device__ __forceinline__ void load_sigt(const SweepArgs& a, float* s_sigt) {
    for (int m = threadIdx.x; m < 256; m += blockDim.x) s_sigt[m] = (m < a.Nm) ? a.sigt[m] : 0.f;
    __syncthreads();
}

// ---------------------------------------------------------------------------------------------
// Level-synchronous schedule: CTA-owned directions, barrier between wavefront levels.
// ---------------------------------------------------------------------------------------------
template <int DPC, int ILP>
__global__ void __launch_bounds__(ILP == 1 ? 1024 : 512) sweep_levels_kernel(SweepArgs a) {
    __shared__ float s_sigt[256];
    load_sigt(a, s_sigt);
    const int nt = blockDim.x;
    for (int d0 = blockIdx.x * DPC; d0 < a.NI; d0 += gridDim.x * DPC) {
        int nl[DPC], lb[DPC];
        float4 dir[DPC];
        int nlmax = 0;
#pragma unroll
        for (int d = 0; d < DPC; ++d) {
            const int i = d0 + d;
            nl[d] = (i < a.NI) ? __ldg(&a.nlev[i]) : 0;
            lb[d] = (i < a.NI) ? __ldg(&a.lvl_base[i]) : 0;
            dir[d] = (i < a.NI) ? __ldg(&a.dirs[i]) : make_float4(0.f, 0.f, 0.f, 0.f);
            nlmax = max(nlmax, nl[d]);
        }
        for (int L = 0; L < nlmax; ++L) {
#pragma unroll
            for (int d = 0; d < DPC; ++d) {
                if (L >= nl[d]) continue;
                const int i = d0 + d;
                const int s0 = __ldg(&a.lvl_start[lb[d] + L]);
                const int s1 = __ldg(&a.lvl_start[lb[d] + L + 1]);
                const int* it = a.items + (size_t)i * a.NE;
                float* base = a.psi + (size_t)i * (size_t)a.NENK;
                for (int es = s0 + threadIdx.x; es < s1; es += nt * ILP) {
                    int item[ILP];
                    bool has[ILP];
#pragma unroll
                    for (int u = 0; u < ILP; ++u) {
                        has[u] = (es + u * nt) < s1;
                        item[u] = has[u] ? __ldcs(&it[es + u * nt]) : 0;
                    }
                    Update up[ILP];
#pragma unroll
                    for (int u = 0; u < ILP; ++u)
                        if (has[u]) assemble<false>(a, base, dir[d], item[u], s_sigt, up[u]);
#pragma unroll
                    for (int u = 0; u < ILP; ++u)
                        if (has[u]) finish<false>(base, item[u], up[u]);
                }
            }
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Dataflow schedule: global chunk queue with bounded waits on per-level completion counters.
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) sweep_dataflow_kernel(SweepArgs a) {
    __shared__ float s_sigt[256];
    load_sigt(a, s_sigt);
    const int lane = threadIdx.x & 31;
    while (true) {
        int cidx = 0;
        if (lane == 0) cidx = atomicAdd(&a.status->work, 1);
        cidx = __shfl_sync(0xffffffffu, cidx, 0);
        if (cidx >= a.nchunks) break;
        const int4 ch = __ldg(&a.chunks[cidx]);
        const int i = ch.x & 0xFFFFFF;
        const int n = ((ch.x >> 24) & 31) + 1;
        int ok = 1;
        if (lane == 0) {
            if (ch.w > 0) {
                const int* ctr = a.done + (ch.z - 1);
                long long spins = 0;
                while (ld_acquire(ctr) < ch.w) {
                    if (++spins > a.spin_limit || *((volatile int*)&a.status->abort)) { ok = 0; break; }
                    __nanosleep(64);
                }
                if (!ok && atomicExch(&a.status->abort, 1) == 0) {
                    a.status->err = LB_ERR_TIMEOUT;
                    a.status->err_chunk = cidx;
                }
            }
            if (*((volatile int*)&a.status->abort)) ok = 0;
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (!ok) break;
        // lane 0's acquire is carried to the other lanes by the warp barrier
        __syncwarp();
        const float4 dir = __ldg(&a.dirs[i]);
        float* base = a.psi + (size_t)i * (size_t)a.NENK;
        if (lane < n) {
            const int item = __ldg(&a.items[(size_t)i * a.NE + ch.y + lane]);
            Update u;
            assemble<true>(a, base, dir, item, s_sigt, u);
            finish<true>(base, item, u);
        }
        __syncwarp();
        if (lane == 0) {
            __threadfence();
            atomicAdd(a.done + ch.z, n);
        }
    }
}

struct Config {
    int kind;      // 0 levels, 1 dataflow
    int threads;
    int dpc;
    int ilp;
};

const Config kConfigs[] = {
    {0, 512, 1, 1}, {0, 512, 1, 2}, {0, 768, 1, 1}, {0, 640, 1, 1}, {0, 1024, 1, 1},
    {0, 256, 1, 2}, {0, 512, 2, 1}, {0, 512, 2, 2}, {0, 1024, 2, 1}, {1, 256, 0, 0},
};
constexpr int kNumConfigs = sizeof(kConfigs) / sizeof(kConfigs[0]);

template <int DPC, int ILP>
cudaError_t launch_levels(const SweepArgs& a, int threads, int sm_count, cudaStream_t s) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sweep_levels_kernel<DPC, ILP>, threads, 0);
    if (per_sm < 1) per_sm = 1;
    int ctas = (a.NI + DPC - 1) / DPC;
    int grid = std::min(ctas, sm_count * per_sm);
    sweep_levels_kernel<DPC, ILP><<<grid, threads, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace

int launch_sweep(Handle* h, float* psi) {
    SweepArgs a;
    a.items = h->d_items;
    a.chunks = h->d_chunks;
    a.lvl_start = h->d_lvl_start;
    a.lvl_base = h->d_lvl_base;
    a.nlev = h->d_nlev;
    a.done = h->d_done;
    a.geom = h->d_geom;
    a.dirs = h->d_dirs;
    a.sigt = h->d_sigt;
    a.psi = psi;
    a.NENK = h->NENK;
    a.NE = h->NE;
    a.NI = h->NI;
    a.nchunks = h->nchunks;
    a.Nm = h->Nm;
    a.status = h->d_status;
    // about a second of polling with 64-ns naps before a wait is declared stuck
    a.spin_limit = 1LL << 24;

    if (h->sweep_cfg_forced < 0) {
        const char* env = std::getenv("LB_SWEEP_CONFIG");
        h->sweep_cfg_forced = (env && *env) ? std::atoi(env) : kNumConfigs;
        if (h->sweep_cfg_forced < 0) h->sweep_cfg_forced = kNumConfigs;
    }
    int cfg_idx;
    bool tuning = false;
    if (h->sweep_cfg_forced < kNumConfigs) cfg_idx = h->sweep_cfg_forced;
    else if (h->sweep_cfg >= 0) cfg_idx = h->sweep_cfg;
    else { cfg_idx = h->sweep_trial; tuning = true; }
    const Config cfg = kConfigs[cfg_idx];

    cudaError_t e = cudaSuccess;
    if (cfg.kind == 1) {
        e = cudaMemsetAsync(h->d_done, 0, sizeof(int) * (size_t)h->total_levels, h->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(h->d_status, 0, sizeof(SweepStatus), h->stream);
        if (e != cudaSuccess) return cuda_fail(h, e, "sweep: reset counters");
    }
    Timer t;
    timer_begin(h, LB_T_SWEEP, t);
    if (cfg.kind == 1) {
        static int df_per_sm = -1;
        if (df_per_sm < 0) {
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&df_per_sm, sweep_dataflow_kernel, 256, 0);
            if (df_per_sm < 1) df_per_sm = 1;
        }
        sweep_dataflow_kernel<<<h->sm_count * df_per_sm, 256, 0, h->stream>>>(a);
        e = cudaGetLastError();
    } else if (cfg.dpc == 1 && cfg.ilp == 1) e = launch_levels<1, 1>(a, cfg.threads, h->sm_count, h->stream);
    else if (cfg.dpc == 1 && cfg.ilp == 2) e = launch_levels<1, 2>(a, cfg.threads, h->sm_count, h->stream);
    else if (cfg.dpc == 2 && cfg.ilp == 1) e = launch_levels<2, 1>(a, cfg.threads, h->sm_count, h->stream);
    else e = launch_levels<2, 2>(a, cfg.threads, h->sm_count, h->stream);
    timer_end(h, t);
    if (e != cudaSuccess) return cuda_fail(h, e, "sweep kernel launch");
    if (cfg.kind == 1) {
        SweepStatus st;
        e = cudaMemcpyAsync(&st, h->d_status, sizeof(st), cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) return cuda_fail(h, e, "sweep kernel");
        if (st.err) {
            char buf[160];
            std::snprintf(buf, sizeof buf, "sweep: dependency wait timed out at chunk %d", st.err_chunk);
            return fail(h, LB_ERR_TIMEOUT, buf);
        }
    }
    if (tuning) {
        e = cudaEventSynchronize(t.b);
        if (e != cudaSuccess) return cuda_fail(h, e, "sweep kernel");
        float ms = 0.f;
        cudaEventElapsedTime(&ms, t.a, t.b);
        h->sweep_trial_ms.push_back(ms);
        if (++h->sweep_trial >= kNumConfigs) {
            int best = 0;
            for (int c = 1; c < kNumConfigs; ++c)
                if (h->sweep_trial_ms[c] < h->sweep_trial_ms[best]) best = c;
            h->sweep_cfg = best;
            const char* verbose = std::getenv("LB_SWEEP_VERBOSE");
            if (verbose && *verbose == '1')
                for (int c = 0; c < kNumConfigs; ++c)
                    std::fprintf(stderr, "sweep config %d (kind %d threads %d dpc %d ilp %d): %.3f ms%s\n", c,
                                 kConfigs[c].kind, kConfigs[c].threads, kConfigs[c].dpc, kConfigs[c].ilp,
                                 h->sweep_trial_ms[c], c == best ? "  <- chosen" : "");
        }
    }
    return LB_OK;
}

int sweep_config(Handle* h, int* kind, int* threads, int* dpc, int* ilp) {
    int c = h->sweep_cfg_forced >= 0 && h->sweep_cfg_forced < kNumConfigs ? h->sweep_cfg_forced : h->sweep_cfg;
    if (c < 0) return -1;
    *kind = kConfigs[c].kind; *threads = kConfigs[c].threads; *dpc = kConfigs[c].dpc; *ilp = kConfigs[c].ilp;
    return c;
}

}  // namespace lb

// =============================================================================================
//  Allocation-free sweep.
//
//  For callers that cannot allocate device memory at solve time: code running inside a host
//  framework that owns the device allocator (a memory pool, a Fortran runtime that only hands out
//  pre-allocated device arrays), or a real-time loop where cudaMalloc's implicit device
//  synchronisation is not acceptable.  The caller passes its own FP32 angular vector; the
//  dataflow schedule's per-level completion counters and status word live in the file-scope array
//  below instead of handle memory, so a call makes no cudaMalloc / cudaFree.
//
//  Limits and sharing: the array holds kNoAllocMaxLevels (direction, level) counters (1 MiB); a
//  problem with more levels is rejected.  Every GPU that loads this library keeps the array until
//  the process exits.  All calls on a device share it and it keeps the last call's contents: the
//  counters are cleared at the start of every call, and calls that overlap on the GPU (two streams,
//  two handles on one device) race on it and must be serialised by the caller.
// =============================================================================================
namespace lb {
namespace {

constexpr int kNoAllocMaxLevels = 1 << 18;
constexpr int kNoAllocStatusInts = 8;   // SweepStatus, padded
static __device__ __align__(256) int g_noalloc_scratch[kNoAllocStatusInts + kNoAllocMaxLevels];

constexpr int kMaxDevices = 64;
void* g_noalloc_ptr[kMaxDevices] = {};

}  // namespace
}  // namespace lb

extern "C" int lb_transport_inv_noalloc(lb_handle* hh, float* psi) {
    using namespace lb;
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || !psi) return LB_ERR_ARG;
    if (h->device < 0) return fail(h, LB_ERR_STATE, "host-only handle: no device attached");
    if (!h->mesh_ready || !h->angle_ready || h->sigt.empty())
        return fail(h, LB_ERR_STATE, "TransportOp%MatInv was called, but the operator was not ready.");
    if (h->total_levels > kNoAllocMaxLevels) {
        char buf[200];
        std::snprintf(buf, sizeof buf,
                      "lb_transport_inv_noalloc: the schedule has %d (direction, level) pairs; the allocation-free "
                      "entry point holds at most %d",
                      h->total_levels, kNoAllocMaxLevels);
        return fail(h, LB_ERR_ARG, buf);
    }
    if (h->device >= kMaxDevices) return fail(h, LB_ERR_ARG, "lb_transport_inv_noalloc: device index too large");
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return cuda_fail(h, e, "lb_transport_inv_noalloc: set device");
    // once per device, with that device current: the device address of the scratch array
    if (!g_noalloc_ptr[h->device]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) return cuda_fail(h, e, "lb_transport_inv_noalloc: scratch address");
        g_noalloc_ptr[h->device] = p;
    }
    int* base = static_cast<int*>(g_noalloc_ptr[h->device]);
    SweepArgs a;
    a.items = h->d_items;
    a.chunks = h->d_chunks;
    a.lvl_start = h->d_lvl_start;
    a.lvl_base = h->d_lvl_base;
    a.nlev = h->d_nlev;
    a.done = base + kNoAllocStatusInts;
    a.geom = h->d_geom;
    a.dirs = h->d_dirs;
    a.sigt = h->d_sigt;
    a.psi = psi;
    a.NENK = h->NENK;
    a.NE = h->NE;
    a.NI = h->NI;
    a.nchunks = h->nchunks;
    a.Nm = h->Nm;
    a.status = reinterpret_cast<SweepStatus*>(base);
    a.spin_limit = 1LL << 24;
    e = cudaMemsetAsync(base, 0, sizeof(int) * ((size_t)kNoAllocStatusInts + h->total_levels), h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "lb_transport_inv_noalloc: clear scratch");
    static int per_sm = -1;
    if (per_sm < 0) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sweep_dataflow_kernel, 256, 0);
        if (per_sm < 1) per_sm = 1;
    }
    sweep_dataflow_kernel<<<h->sm_count * per_sm, 256, 0, h->stream>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(h, e, "lb_transport_inv_noalloc: launch");
    SweepStatus st;
    e = cudaMemcpyAsync(&st, base, sizeof(st), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "lb_transport_inv_noalloc: sweep");
    if (st.err) {
        char buf[160];
        std::snprintf(buf, sizeof buf, "sweep: dependency wait timed out at chunk %d", st.err_chunk);
        return fail(h, LB_ERR_TIMEOUT, buf);
    }
    return LB_OK;
}
