// Persistent discontinuous-Galerkin upwind sweep for linear tetrahedra, FP32, sm_100a.
//
// Replaces TransportAlgebra.f90:29-246 (Sweep + ApplyInvertedDiagonal + LocalLU) and the
// EncodeSweep.f90 permutations around it.  One thread performs one element-direction update;
// a warp takes a chunk of up to 32 consecutive elements of one wavefront level of one direction.
// Chunks are claimed from a global counter in level-major order across all directions; a chunk
// waits (bounded) on the completion counter of the previous level of its own direction, so all
// NI directions sweep concurrently through their own wavefronts.
//
// Element operator.  For linear tets the mass-eliminated matrices of
// FiniteElementAnalysis.f90:228-304 have closed forms in terms of the scaled face vectors
// s_f = A_f n_f / V (area, outward unit normal, volume).  With c_f = k . s_f:
//   -sum_d k_d IC_d (k,kp) = (5/3) c_{3-k}                  (face 3-k is opposite vertex k)
//   (k.n_f) IFM_f (k,kp) = c_f P_f(k,kp),   P_f(k,kp) = [kp in f] * (k==kp ? 2 : k in f ? 1/3 : -4/3)
//   (k.n_f) IIM_f = c_f P_f with columns mapped to the neighbour's local nodes.
// so the 4x4 system  T = sigma I - sum_d k_d IC_d + sum_{f: k.n_f >= 0} (k.n_f) IFM_f  and the
// upstream coupling  rhs -= sum_{f upstream} (k.n_f) IIM_f psi_up  are assembled from 12 floats
// per element.  The system is solved by Gaussian elimination with row pivoting (LocalLU).
#include "lb_internal.h"
#include <cstdio>

namespace lb {

namespace {

constexpr float kThird = 1.0f / 3.0f;
constexpr float kFiveThirds = 5.0f / 3.0f;
constexpr float kFourThirds = 4.0f / 3.0f;

struct SweepArgs {
    const int* __restrict__ items;
    const int4* __restrict__ chunks;
    int* done;
    const float4* __restrict__ geom;
    const float4* __restrict__ dirs;
    const float* __restrict__ sigt;
    float* psi;
    long long NENK;
    int NE;
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

__device__ __forceinline__ float4 ld_cg4(const float* p) {
    return __ldcg(reinterpret_cast<const float4*>(p));
}

__device__ __forceinline__ float pick(const float4& v, int idx) {
    float r = v.x;
    r = (idx == 1) ? v.y : r;
    r = (idx == 2) ? v.z : r;
    r = (idx == 3) ? v.w : r;
    return r;
}

// Gaussian elimination with row pivoting on a 4x4 system, registers only.  The pivot is the first
// row holding the largest |A(r,k)| (strict '>' comparison, as LocalLU).
__device__ __forceinline__ void solve4(float A[4][4], float b[4]) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float best = fabsf(A[k][k]);
        int p = k;
#pragma unroll
        for (int r = k + 1; r < 4; ++r) {
            float v = fabsf(A[r][k]);
            if (v > best) { best = v; p = r; }
        }
#pragma unroll
        for (int r = k + 1; r < 4; ++r) {
            if (p == r) {
#pragma unroll
                for (int c = 0; c < 4; ++c) { float t = A[k][c]; A[k][c] = A[r][c]; A[r][c] = t; }
                float t = b[k]; b[k] = b[r]; b[r] = t;
            }
        }
        float inv = 1.0f / A[k][k];
#pragma unroll
        for (int r = k + 1; r < 4; ++r) {
            float f = A[r][k] * inv;
#pragma unroll
            for (int c = k + 1; c < 4; ++c) A[r][c] = fmaf(-f, A[k][c], A[r][c]);
            b[r] = fmaf(-f, b[k], b[r]);
        }
    }
    b[3] = b[3] / A[3][3];
#pragma unroll
    for (int i = 2; i >= 0; --i) {
        float x = b[i];
#pragma unroll
        for (int j = i + 1; j < 4; ++j) x = fmaf(-A[i][j], b[j], x);
        b[i] = x / A[i][i];
    }
}

__device__ __forceinline__ void element_update(const SweepArgs& a, int i, float4 dir, int item, const float* s_sigt) {
    const int e = item & 0xFFFFFF;
    const int upm = (item >> 24) & 0xF;
    const int outm = (item >> 28) & 0xF;
    const float4 gx = __ldg(&a.geom[(size_t)e * 4 + 0]);
    const float4 gy = __ldg(&a.geom[(size_t)e * 4 + 1]);
    const float4 gz = __ldg(&a.geom[(size_t)e * 4 + 2]);
    const int4 gn = __ldg(reinterpret_cast<const int4*>(&a.geom[(size_t)e * 4 + 3]));
    float c[4];
    c[0] = fmaf(dir.x, gx.x, fmaf(dir.y, gy.x, dir.z * gz.x));
    c[1] = fmaf(dir.x, gx.y, fmaf(dir.y, gy.y, dir.z * gz.y));
    c[2] = fmaf(dir.x, gx.z, fmaf(dir.y, gy.z, dir.z * gz.z));
    c[3] = fmaf(dir.x, gx.w, fmaf(dir.y, gy.w, dir.z * gz.w));
    const unsigned nw[4] = {(unsigned)gn.x, (unsigned)gn.y, (unsigned)gn.z, (unsigned)gn.w};
    const int matid = (int)((nw[0] >> 30) | ((nw[1] >> 30) << 2) | ((nw[2] >> 30) << 4) | ((nw[3] >> 30) << 6));
    const float sig = s_sigt[matid];

    float* base = a.psi + (size_t)i * (size_t)a.NENK;
    const float4 q = ld_cg4(base + 4 * (size_t)e);
    float rhs[4] = {q.x, q.y, q.z, q.w};

    // face -> local nodes (gmsh order) and opposite vertex
    constexpr int F[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        if ((upm >> f) & 1) {
            const unsigned wd = nw[f];
            const int ep = (int)(wd & 0xFFFFFFu);
            const float4 u4 = ld_cg4(base + 4 * (size_t)ep);
            const float u0 = pick(u4, (wd >> 24) & 3);
            const float u1 = pick(u4, (wd >> 26) & 3);
            const float u2 = pick(u4, (wd >> 28) & 3);
            const float U = u0 + u1 + u2;
            const float cf = c[f];
            const float t3 = U * kThird;
            rhs[F[f][0]] = fmaf(-cf, fmaf(kFiveThirds, u0, t3), rhs[F[f][0]]);
            rhs[F[f][1]] = fmaf(-cf, fmaf(kFiveThirds, u1, t3), rhs[F[f][1]]);
            rhs[F[f][2]] = fmaf(-cf, fmaf(kFiveThirds, u2, t3), rhs[F[f][2]]);
            rhs[3 - f] = fmaf(cf * kFourThirds, U, rhs[3 - f]);
        }
    }

    float A[4][4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float g = kFiveThirds * c[3 - k];
#pragma unroll
        for (int kp = 0; kp < 4; ++kp) A[k][kp] = (k == kp) ? sig + g : g;
    }
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        const float cf = ((outm >> f) & 1) ? c[f] : 0.0f;
#pragma unroll
        for (int jj = 0; jj < 3; ++jj) {
            const int kp = F[f][jj];
#pragma unroll
            for (int ii = 0; ii < 3; ++ii) {
                const int k = F[f][ii];
                A[k][kp] = fmaf(cf, (k == kp) ? 2.0f : kThird, A[k][kp]);
            }
            A[3 - f][kp] = fmaf(-cf, kFourThirds, A[3 - f][kp]);
        }
    }
    solve4(A, rhs);
    __stcg(reinterpret_cast<float4*>(base + 4 * (size_t)e), make_float4(rhs[0], rhs[1], rhs[2], rhs[3]));
}

__global__ void __launch_bounds__(256) sweep_kernel(SweepArgs a) {
    __shared__ float s_sigt[256];
    for (int m = threadIdx.x; m < 256; m += blockDim.x) s_sigt[m] = (m < a.Nm) ? a.sigt[m] : 0.f;
    __syncthreads();
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
        if (lane < n) {
            const int item = __ldg(&a.items[(size_t)i * a.NE + ch.y + lane]);
            element_update(a, i, dir, item, s_sigt);
        }
        __syncwarp();
        if (lane == 0) {
            __threadfence();
            atomicAdd(a.done + ch.z, n);
        }
    }
}

}  // namespace

int launch_sweep(Handle* h, float* psi) {
    static int blocks_per_sm = -1;
    if (blocks_per_sm < 0) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, sweep_kernel, 256, 0);
        if (blocks_per_sm < 1) blocks_per_sm = 1;
    }
    SweepArgs a;
    a.items = h->d_items;
    a.chunks = h->d_chunks;
    a.done = h->d_done;
    a.geom = h->d_geom;
    a.dirs = h->d_dirs;
    a.sigt = h->d_sigt;
    a.psi = psi;
    a.NENK = h->NENK;
    a.NE = h->NE;
    a.nchunks = h->nchunks;
    a.Nm = h->Nm;
    a.status = h->d_status;
    // about a second of polling with 64-ns naps before a wait is declared stuck
    a.spin_limit = 1LL << 24;
    cudaError_t e;
    e = cudaMemsetAsync(h->d_done, 0, sizeof(int) * (size_t)h->total_levels, h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "sweep: reset counters");
    e = cudaMemsetAsync(h->d_status, 0, sizeof(SweepStatus), h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "sweep: reset status");
    Timer t;
    timer_begin(h, LB_T_SWEEP, t);
    int grid = h->sm_count * blocks_per_sm;
    sweep_kernel<<<grid, 256, 0, h->stream>>>(a);
    timer_end(h, t);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(h, e, "sweep kernel launch");
    SweepStatus st;
    e = cudaMemcpyAsync(&st, h->d_status, sizeof(st), cudaMemcpyDeviceToHost, h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "sweep: read status");
    e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "sweep kernel");
    if (st.err) {
        char buf[160];
        std::snprintf(buf, sizeof buf, "sweep: dependency wait timed out at chunk %d", st.err_chunk);
        return fail(h, LB_ERR_TIMEOUT, buf);
    }
    return LB_OK;
}

}  // namespace lb
