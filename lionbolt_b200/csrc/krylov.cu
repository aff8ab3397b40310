// FP64 vector kernels for the flux-moment Krylov solvers (GMRES/FGMRES/SI) and the multigroup
// source / dose tallies.  The reference runs these as serial Fortran loops inside SPARSKIT
// (third_party/SPARSKIT/iters.f: gmres :1901-2206, mgsro :3465-3587) and Main.f90.
// Reductions are deterministic: fixed grid, per-block partials summed on the host in block order.
#include "lb_internal.h"
#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>

namespace lb {

namespace {

constexpr int kMaxDots = 32;
constexpr int kRedThreads = 256;

struct Coefs { double c[kMaxDots]; };

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

constexpr int kPartStride = kMaxDots + 1;   // partial row: NV dots + the squared norm

// Loads in flight per thread: small NV unrolls the element loop instead.
template <int NV>
__host__ __device__ constexpr int unroll_for() { return NV < 2 ? 4 : (NV < 6 ? 2 : 1); }

// Block-level reduction of acc[0..NV] into partial[blockIdx.x][0..NV].
template <int NV>
__device__ __forceinline__ void block_reduce_store(double (&acc)[NV + 1], double* partial) {
    __shared__ double s[kRedThreads / 32][NV + 1];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int j = 0; j <= NV; ++j) {
        const double v = warp_sum(acc[j]);
        if (lane == 0) s[warp][j] = v;
    }
    __syncthreads();
    if (threadIdx.x <= NV) {
        double v = 0.0;
#pragma unroll
        for (int k = 0; k < kRedThreads / 32; ++k) v += s[k][threadIdx.x];
        partial[(size_t)blockIdx.x * kPartStride + threadIdx.x] = v;
    }
}

// partial[b][j] = V_j . w (j < NV) and partial[b][NV] = w . w over this block's elements.
// Vectors are read as double2 (n is even: n = nm * NENK with NENK a multiple of 4).
// ZM: the vector passed is z and w = V_{NV-1} - z (the Arnoldi step's A v = v - z formed here, from the basis
// vector this pass reads anyway, instead of in the D2M epilogue).
template <int NV, bool ZM = false>
__global__ void __launch_bounds__(kRedThreads) dots_t(const double* __restrict__ V, size_t ldv,
                                                     const double* __restrict__ w, size_t n2, double* partial) {
    constexpr int U = unroll_for<NV>();
    double acc[NV + 1];
#pragma unroll
    for (int j = 0; j <= NV; ++j) acc[j] = 0.0;
    const double2* w2 = reinterpret_cast<const double2*>(w);
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t q0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q0 < n2; q0 += U * stride) {
        double2 wq[U], v[U][NV > 0 ? NV : 1];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const size_t q = q0 + u * stride;
            const bool in = q < n2;
            wq[u] = in ? __ldcs(w2 + q) : make_double2(0.0, 0.0);
#pragma unroll
            for (int j = 0; j < NV; ++j)
                v[u][j] = in ? __ldcs(reinterpret_cast<const double2*>(V + (size_t)j * ldv) + q) : make_double2(0.0, 0.0);
            if constexpr (ZM) wq[u] = make_double2(v[u][NV - 1].x - wq[u].x, v[u][NV - 1].y - wq[u].y);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
#pragma unroll
            for (int j = 0; j < NV; ++j) acc[j] = fma(v[u][j].x, wq[u].x, fma(v[u][j].y, wq[u].y, acc[j]));
            acc[NV] = fma(wq[u].x, wq[u].x, fma(wq[u].y, wq[u].y, acc[NV]));
        }
    }
    block_reduce_store<NV>(acc, partial);
}

// w <- w - sum_j c_j V_j; partial[b][j] = V_j . w_new (j < NV, when DOTS) and partial[b][NV] =
// w_new . w_new.  Up to 16 vectors stay in registers between the update and the dots; beyond that
// the dots re-read the block's elements (L1/L2 hits).
// ZM: w holds z on entry and the vector updated is V_{NV-1} - z (see dots_t).
template <int NV, bool DOTS, bool ZM = false>
__global__ void __launch_bounds__(kRedThreads) axpy_dots_t(double* w, const double* __restrict__ V, size_t ldv, Coefs cf,
                                                          size_t n2, double* partial) {
    double acc[NV + 1];
#pragma unroll
    for (int j = 0; j <= NV; ++j) acc[j] = 0.0;
    double2* w2 = reinterpret_cast<double2*>(w);
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n2; q += stride) {
        double2 x = w2[q];
        if constexpr (NV <= 16) {
            double2 v[NV > 0 ? NV : 1];
#pragma unroll
            for (int j = 0; j < NV; ++j) v[j] = __ldg(reinterpret_cast<const double2*>(V + (size_t)j * ldv) + q);
            if constexpr (ZM) x = make_double2(v[NV - 1].x - x.x, v[NV - 1].y - x.y);
#pragma unroll
            for (int j = 0; j < NV; ++j) {
                x.x = fma(-cf.c[j], v[j].x, x.x);
                x.y = fma(-cf.c[j], v[j].y, x.y);
            }
            w2[q] = x;
            if constexpr (DOTS) {
#pragma unroll
                for (int j = 0; j < NV; ++j) acc[j] = fma(v[j].x, x.x, fma(v[j].y, x.y, acc[j]));
            }
        } else {
            if constexpr (ZM) {
                const double2 vl = __ldg(reinterpret_cast<const double2*>(V + (size_t)(NV - 1) * ldv) + q);
                x = make_double2(vl.x - x.x, vl.y - x.y);
            }
#pragma unroll
            for (int j = 0; j < NV; ++j) {
                const double2 v = __ldg(reinterpret_cast<const double2*>(V + (size_t)j * ldv) + q);
                x.x = fma(-cf.c[j], v.x, x.x);
                x.y = fma(-cf.c[j], v.y, x.y);
            }
            w2[q] = x;
            if constexpr (DOTS) {
#pragma unroll
                for (int j = 0; j < NV; ++j) {
                    const double2 v = __ldg(reinterpret_cast<const double2*>(V + (size_t)j * ldv) + q);
                    acc[j] = fma(v.x, x.x, fma(v.y, x.y, acc[j]));
                }
            }
        }
        acc[NV] = fma(x.x, x.x, fma(x.y, x.y, acc[NV]));
    }
    block_reduce_store<NV>(acc, partial);
}

// w <- (w - sum_j c_j V_j) * scale
template <int NV>
__global__ void __launch_bounds__(kRedThreads) axpy_scale_t(double* w, const double* __restrict__ V, size_t ldv, Coefs cf,
                                                           double scale, size_t n2) {
    double2* w2 = reinterpret_cast<double2*>(w);
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n2; q += stride) {
        double2 x = w2[q];
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            const double2 v = __ldcs(reinterpret_cast<const double2*>(V + (size_t)j * ldv) + q);
            x.x = fma(-cf.c[j], v.x, x.x);
            x.y = fma(-cf.c[j], v.y, x.y);
        }
        x.x *= scale;
        x.y *= scale;
        w2[q] = x;
    }
}

// y <- a x + b y; partial[b][0] = y . y
__global__ void __launch_bounds__(kRedThreads) axpby_norm_kernel(double* y, const double* __restrict__ x, double a, double b,
                                                                size_t n2, double* partial) {
    double acc[1] = {0.0};
    double2* y2 = reinterpret_cast<double2*>(y);
    const double2* x2 = reinterpret_cast<const double2*>(x);
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n2; q += stride) {
        const double2 u = __ldcs(x2 + q);
        double2 v = y2[q];
        v.x = a * u.x + b * v.x;
        v.y = a * u.y + b * v.y;
        y2[q] = v;
        acc[0] = fma(v.x, v.x, fma(v.y, v.y, acc[0]));
    }
    block_reduce_store<0>(acc, partial);
}

// Compile-time dispatch of nv in [0, kMaxDots].
template <int N>
struct NvDispatch {
    template <class F>
    static void run(int nv, F&& f) {
        if (nv == N) f(std::integral_constant<int, N>{});
        else NvDispatch<N - 1>::run(nv, f);
    }
};
template <>
struct NvDispatch<-1> {
    template <class F>
    static void run(int, F&&) {}
};

// Resident blocks per SM of a kernel (cached per instantiation).
template <class K>
int blocks_per_sm(K kernel) {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, kRedThreads, 0) != cudaSuccess) {
        cudaGetLastError();
        b = 1;
    }
    return b < 1 ? 1 : b;
}

__global__ void axpby_kernel(double* y, const double* x, double a, double b, size_t n) {
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
        y[q] = a * x[q] + b * y[q];
}

__global__ void scale_kernel(double* y, double a, size_t n) {
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) y[q] *= a;
}

// z[j][n] = c[j] v[j][n] for the nm moment rows (blockIdx.y = j)
struct RowCoefs {
    double c[kMaxRowCoefs];
};
__global__ void scale_rows_kernel(double* __restrict__ z, const double* __restrict__ v, RowCoefs rc, size_t NENK) {
    const double c = rc.c[blockIdx.y];
    const size_t off = (size_t)blockIdx.y * NENK;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < NENK; q += (size_t)gridDim.x * blockDim.x)
        z[off + q] = c * v[off + q];
}

__global__ void fill_kernel(double* y, double v, size_t n) {
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) y[q] = v;
}

__global__ void f64_to_f32_kernel(float* y, const double* x, size_t n) {
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
        y[q] = (float)x[q];
}

__global__ void f32_to_f64_kernel(double* y, const float* x, size_t n) {
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
        y[q] = (double)x[q];
}

// src[j][n] (+)= sigl[mat(n)][j] * phi[j][n]
__global__ void moment_source_kernel(double* src, const double* __restrict__ phi, const float* __restrict__ sigl,
                                     const int* __restrict__ mat, long long NENK, int nm, int nmpad, int accumulate) {
    const size_t total = (size_t)nm * NENK;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(q / NENK);
        const long long n = (long long)(q % NENK);
        const double v = (double)sigl[(size_t)mat[n >> 2] * nmpad + j] * phi[q];
        src[q] = accumulate ? src[q] + v : v;
    }
}

// src[j][n] += sigl[mat(n)][j] * ybeam[j] * unc[n]   (first-collision source of a beam)
__global__ void unc_source_kernel(double* src, const double* __restrict__ unc, const double* __restrict__ ybeam,
                                  const float* __restrict__ sigl, const int* __restrict__ mat, long long NENK, int nm,
                                  int nmpad) {
    const size_t total = (size_t)nm * NENK;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(q / NENK);
        const long long n = (long long)(q % NENK);
        src[q] += (double)sigl[(size_t)mat[n >> 2] * nmpad + j] * ybeam[j] * unc[n];
    }
}

// Group source in one pass (Main.f90 PIEISource :544-747 restated in moment space):
//   src[j][n] = sum_{g' < g} sigma_{g'->g}(mat(n), l(j)) phi_{g'}[j][n]
//             + sigma_{0->g}(mat(n), l(j)) Y_j(Omega_beam) unc[n]
// tab = transfer tables [G][G][Nm][nmpad]; phi_all = [G][nm][NENK] solved group moments.
__global__ void __launch_bounds__(256) group_source_kernel(double* __restrict__ src, const double* __restrict__ phi_all,
                                                          const float* __restrict__ tab, int G, int g,
                                                          const double* __restrict__ unc,
                                                          const double* __restrict__ ybeam, const int* __restrict__ mat,
                                                          long long NENK, int Nm, int nm, int nmpad) {
    // One element (its four DG nodes, one material) per thread: one table entry per (g', j) for four nodes,
    // and 32-byte loads, so a warp reads 1 KB of one moment row at a time.  Each node sums g' = 0, 1, ...
    // in the same order as a node-per-thread loop.
    const size_t nvec = (size_t)nm * NENK;
    const size_t tstride = (size_t)G * Nm * nmpad;   // g' -> g' + 1 in the (g', g, m, j) table
    const long long NE = NENK >> 2;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < NE; e += (long long)gridDim.x * blockDim.x) {
        const long long n = e << 2;
        const int m = mat[e];
        const double4 u = unc ? *reinterpret_cast<const double4*>(unc + n) : make_double4(0.0, 0.0, 0.0, 0.0);
        const float* t0 = tab + ((size_t)g * Nm + m) * nmpad;   // (g' = 0, g)
        for (int j = 0; j < nm; ++j) {
            const double y = (double)t0[j] * ybeam[j];
            double a0 = y * u.x, a1 = y * u.y, a2 = y * u.z, a3 = y * u.w;
            const float* tp = t0 + j;
            const double* pp = phi_all + (size_t)j * NENK + n;
            for (int gp = 0; gp < g; ++gp) {
                const double t = (double)tp[(size_t)gp * tstride];
                const double4 p = *reinterpret_cast<const double4*>(pp + (size_t)gp * nvec);
                a0 += t * p.x;
                a1 += t * p.y;
                a2 += t * p.z;
                a3 += t * p.w;
            }
            *reinterpret_cast<double4*>(src + (size_t)j * NENK + n) = make_double4(a0, a1, a2, a3);
        }
    }
}

// scalar fluence fl = sqrt(4 pi) phi_00 + s*unc; flux = fl; dose += dd[mat] fl (TallyDeposition.f90:19)
__global__ void dose_kernel(const double* __restrict__ phi00, const double* __restrict__ unc, double unc_scale,
                            const double* __restrict__ dd, const int* __restrict__ mat, double* flux, double* dose,
                            long long NENK) {
    const double s4pi = 3.5449077018110320546;   // sqrt(4 pi): phi_00 = fluence / sqrt(4 pi)
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < NENK; n += (long long)gridDim.x * blockDim.x) {
        double fl = s4pi * phi00[n];
        if (unc) fl += unc_scale * unc[n];
        flux[n] = fl;
        dose[n] += dd[mat[n >> 2]] * fl;
    }
}

// ---- segmented (per-problem) versions for batches: block b belongs to the segment whose
// [blk0, blk0 + nblk) contains it; the segment table is small (one entry per problem).
__device__ __forceinline__ int seg_of_block(const SegVec* segs, int nseg) {
    int s = 0;
    while (s + 1 < nseg && (int)blockIdx.x >= segs[s + 1].blk0) ++s;
    return s;
}

template <int NV>
__global__ void __launch_bounds__(kRedThreads) seg_dots_t(const SegVec* __restrict__ segs, int nseg, double* partial) {
    const SegVec S = segs[seg_of_block(segs, nseg)];
    double acc[NV + 1];
#pragma unroll
    for (int j = 0; j <= NV; ++j) acc[j] = 0.0;
    const double2* w2 = reinterpret_cast<const double2*>(S.w);
    const size_t stride = (size_t)S.nblk * blockDim.x;
    for (size_t q = (size_t)(blockIdx.x - S.blk0) * blockDim.x + threadIdx.x; q < S.n2; q += stride) {
        const double2 wq = __ldcs(w2 + q);
        double2 v[NV > 0 ? NV : 1];
#pragma unroll
        for (int j = 0; j < NV; ++j) v[j] = __ldcs(reinterpret_cast<const double2*>(S.V + (size_t)j * S.ldv) + q);
#pragma unroll
        for (int j = 0; j < NV; ++j) acc[j] = fma(v[j].x, wq.x, fma(v[j].y, wq.y, acc[j]));
        acc[NV] = fma(wq.x, wq.x, fma(wq.y, wq.y, acc[NV]));
    }
    block_reduce_store<NV>(acc, partial);
}

template <int NV, bool DOTS>
__global__ void __launch_bounds__(kRedThreads) seg_axpy_dots_t(const SegVec* __restrict__ segs, int nseg,
                                                              const double* __restrict__ coef, double* partial) {
    const SegVec S = segs[seg_of_block(segs, nseg)];
    double c[NV > 0 ? NV : 1];
#pragma unroll
    for (int j = 0; j < NV; ++j) c[j] = coef[S.coef + j];
    double acc[NV + 1];
#pragma unroll
    for (int j = 0; j <= NV; ++j) acc[j] = 0.0;
    double2* w2 = reinterpret_cast<double2*>(S.w);
    const size_t stride = (size_t)S.nblk * blockDim.x;
    for (size_t q = (size_t)(blockIdx.x - S.blk0) * blockDim.x + threadIdx.x; q < S.n2; q += stride) {
        double2 x = w2[q];
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            const double2 v = __ldg(reinterpret_cast<const double2*>(S.V + (size_t)j * S.ldv) + q);
            x.x = fma(-c[j], v.x, x.x);
            x.y = fma(-c[j], v.y, x.y);
        }
        w2[q] = x;
        if constexpr (DOTS) {
#pragma unroll
            for (int j = 0; j < NV; ++j) {
                const double2 v = __ldg(reinterpret_cast<const double2*>(S.V + (size_t)j * S.ldv) + q);
                acc[j] = fma(v.x, x.x, fma(v.y, x.y, acc[j]));
            }
        }
        acc[NV] = fma(x.x, x.x, fma(x.y, x.y, acc[NV]));
    }
    block_reduce_store<NV>(acc, partial);
}

template <int NV>
__global__ void __launch_bounds__(kRedThreads) seg_axpy_scale_t(const SegVec* __restrict__ segs, int nseg,
                                                               const double* __restrict__ coef) {
    const SegVec S = segs[seg_of_block(segs, nseg)];
    double c[NV > 0 ? NV : 1];
#pragma unroll
    for (int j = 0; j < NV; ++j) c[j] = coef[S.coef + j];
    double2* w2 = reinterpret_cast<double2*>(S.w);
    double2* o2 = reinterpret_cast<double2*>(S.w2);
    const size_t stride = (size_t)S.nblk * blockDim.x;
    for (size_t q = (size_t)(blockIdx.x - S.blk0) * blockDim.x + threadIdx.x; q < S.n2; q += stride) {
        double2 x = w2[q];
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            const double2 v = __ldcs(reinterpret_cast<const double2*>(S.V + (size_t)j * S.ldv) + q);
            x.x = fma(-c[j], v.x, x.x);
            x.y = fma(-c[j], v.y, x.y);
        }
        x.x *= S.scale;
        x.y *= S.scale;
        w2[q] = x;
        if (o2) o2[q] = x;
    }
}

__global__ void __launch_bounds__(kRedThreads) seg_axpby_norm_kernel(const SegVec* __restrict__ segs, int nseg,
                                                                    double* partial) {
    const SegVec S = segs[seg_of_block(segs, nseg)];
    double acc[1] = {0.0};
    double2* y2 = reinterpret_cast<double2*>(S.w);
    const double2* x2 = reinterpret_cast<const double2*>(S.x);
    const size_t stride = (size_t)S.nblk * blockDim.x;
    for (size_t q = (size_t)(blockIdx.x - S.blk0) * blockDim.x + threadIdx.x; q < S.n2; q += stride) {
        const double2 u = __ldcs(x2 + q);
        double2 v = y2[q];
        v.x = S.a * u.x + S.b * v.x;
        v.y = S.a * u.y + S.b * v.y;
        y2[q] = v;
        acc[0] = fma(v.x, v.x, fma(v.y, v.y, acc[0]));
    }
    block_reduce_store<0>(acc, partial);
}

inline int grid_for(Handle* h, size_t n) {
    size_t g = (n + 255) / 256;
    size_t cap = (size_t)h->sm_count * 8;
    return (int)std::max<size_t>(1, std::min(g, cap));
}

}  // namespace

// Sum of the per-block partials (block order: deterministic) for entries 0..cnt-1.
static int reduce_partials(Handle* h, int grid, int cnt, double* out) {
    cudaError_t e = cudaMemcpyAsync(h->h_red, h->d_red, sizeof(double) * (size_t)grid * kPartStride,
                                    cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "Krylov reduction");
    for (int j = 0; j < cnt; ++j) {
        double s = 0.0;
        for (int b = 0; b < grid; ++b) s += h->h_red[(size_t)b * kPartStride + j];
        out[j] = s;
    }
    return LB_OK;
}

static bool check_args(Handle* h, int nv, size_t n, const char* what, int* rc) {
    if (nv < 0 || nv > kMaxDots) { *rc = fail(h, LB_ERR_ARG, std::string(what) + ": too many vectors"); return false; }
    if (n % 2) { *rc = fail(h, LB_ERR_ARG, std::string(what) + ": odd vector length"); return false; }
    return true;
}

// out[j] = V_j . w for j < nv; *wnorm2 = w . w (either output may be null).
int k_dots_norm(Handle* h, const double* V, size_t ldv, int nv, const double* w, size_t n, double* out, double* wnorm2,
                bool zm) {
    int rc = 0;
    if (!check_args(h, nv, n, "dots", &rc)) return rc;
    if (zm && nv < 1) return fail(h, LB_ERR_ARG, "dots: the z form needs a basis vector");
    int grid = 0;
    Timer t;
    timer_begin(h, LB_T_KRYLOV, t);
    NvDispatch<kMaxDots>::run(nv, [&](auto c) {
        constexpr int NV = decltype(c)::value;
        if (zm) {
            if constexpr (NV >= 1) {
                static const int occ = blocks_per_sm(dots_t<NV, true>);
                grid = h->sm_count * occ;
                dots_t<NV, true><<<grid, kRedThreads, 0, h->stream>>>(V, ldv, w, n / 2, h->d_red);
            }
        } else {
            static const int occ = blocks_per_sm(dots_t<NV>);
            grid = h->sm_count * occ;
            dots_t<NV><<<grid, kRedThreads, 0, h->stream>>>(V, ldv, w, n / 2, h->d_red);
        }
    });
    timer_end(h, t);
    double tmp[kPartStride];
    if ((rc = reduce_partials(h, grid, nv + 1, tmp))) return rc;
    for (int j = 0; j < nv; ++j)
        if (out) out[j] = tmp[j];
    if (wnorm2) *wnorm2 = tmp[nv];
    return LB_OK;
}

int k_dots(Handle* h, const double* V, size_t ldv, int nv, const double* w, size_t n, double* out) {
    return k_dots_norm(h, V, ldv, nv, w, n, out, nullptr, false);
}

// w -= sum_j coef[j] V_j; then dots[j] = V_j . w (if dots != null) and *nrm2 = w . w (if non-null).
int k_axpy_dots(Handle* h, double* w, const double* V, size_t ldv, int nv, const double* coef, size_t n, double* dots,
                double* nrm2, bool zm) {
    int rc = 0;
    if (!check_args(h, nv, n, "axpy", &rc)) return rc;
    if (zm && (nv < 1 || !dots)) return fail(h, LB_ERR_ARG, "axpy: the z form needs a basis vector and the dots");
    Coefs cf;
    for (int j = 0; j < kMaxDots; ++j) cf.c[j] = (j < nv) ? coef[j] : 0.0;
    int grid = 0;
    Timer t;
    timer_begin(h, LB_T_KRYLOV, t);
    NvDispatch<kMaxDots>::run(nv, [&](auto c) {
        constexpr int NV = decltype(c)::value;
        if (zm) {
            if constexpr (NV >= 1) {
                static const int occ = blocks_per_sm(axpy_dots_t<NV, true, true>);
                grid = h->sm_count * occ;
                axpy_dots_t<NV, true, true><<<grid, kRedThreads, 0, h->stream>>>(w, V, ldv, cf, n / 2, h->d_red);
            }
        } else if (dots) {
            static const int occ = blocks_per_sm(axpy_dots_t<NV, true>);
            grid = h->sm_count * occ;
            axpy_dots_t<NV, true><<<grid, kRedThreads, 0, h->stream>>>(w, V, ldv, cf, n / 2, h->d_red);
        } else {
            static const int occ = blocks_per_sm(axpy_dots_t<NV, false>);
            grid = h->sm_count * occ;
            axpy_dots_t<NV, false><<<grid, kRedThreads, 0, h->stream>>>(w, V, ldv, cf, n / 2, h->d_red);
        }
    });
    timer_end(h, t);
    if (!dots && !nrm2) return LB_OK;
    double tmp[kPartStride];
    if ((rc = reduce_partials(h, grid, nv + 1, tmp))) return rc;
    if (dots)
        for (int j = 0; j < nv; ++j) dots[j] = tmp[j];
    if (nrm2) *nrm2 = tmp[nv];
    return LB_OK;
}

// w <- (w - sum_j coef[j] V_j) * scale
int k_axpy_scale(Handle* h, double* w, const double* V, size_t ldv, int nv, const double* coef, double scale, size_t n) {
    int rc = 0;
    if (!check_args(h, nv, n, "axpy", &rc)) return rc;
    Coefs cf;
    for (int j = 0; j < kMaxDots; ++j) cf.c[j] = (j < nv) ? coef[j] : 0.0;
    Timer t;
    timer_begin(h, LB_T_KRYLOV, t);
    NvDispatch<kMaxDots>::run(nv, [&](auto c) {
        constexpr int NV = decltype(c)::value;
        static const int occ = blocks_per_sm(axpy_scale_t<NV>);
        axpy_scale_t<NV><<<h->sm_count * occ, kRedThreads, 0, h->stream>>>(w, V, ldv, cf, scale, n / 2);
    });
    timer_end(h, t);
    return LB_OK;
}

int k_multi_axpy_norm(Handle* h, double* w, const double* V, size_t ldv, int nv, const double* coef, size_t n, double* nrm2) {
    return k_axpy_dots(h, w, V, ldv, nv, coef, n, nullptr, nrm2);
}

int k_multi_axpy(Handle* h, double* w, const double* V, size_t ldv, int nv, const double* coef, size_t n) {
    return k_axpy_scale(h, w, V, ldv, nv, coef, 1.0, n);
}

// y <- a x + b y and *nrm2 = y . y
int k_axpby_norm(Handle* h, double* y, const double* x, double a, double b, size_t n, double* nrm2) {
    int rc = 0;
    if (!check_args(h, 0, n, "axpby", &rc)) return rc;
    static const int occ = blocks_per_sm(axpby_norm_kernel);
    const int grid = h->sm_count * occ;
    Timer t;
    timer_begin(h, LB_T_KRYLOV, t);
    axpby_norm_kernel<<<grid, kRedThreads, 0, h->stream>>>(y, x, a, b, n / 2, h->d_red);
    timer_end(h, t);
    double tmp[1];
    if ((rc = reduce_partials(h, grid, 1, tmp))) return rc;
    if (nrm2) *nrm2 = tmp[0];
    return LB_OK;
}

int k_axpby(Handle* h, double* y, const double* x, double a, double b, size_t n) {
    Timer t;
    timer_begin(h, LB_T_KRYLOV, t);
    axpby_kernel<<<grid_for(h, n), 256, 0, h->stream>>>(y, x, a, b, n);
    timer_end(h, t);
    return LB_OK;
}

int k_scale(Handle* h, double* y, double a, size_t n) {
    Timer t;
    timer_begin(h, LB_T_KRYLOV, t);
    scale_kernel<<<grid_for(h, n), 256, 0, h->stream>>>(y, a, n);
    timer_end(h, t);
    return LB_OK;
}

int k_copy(Handle* h, double* y, const double* x, size_t n) {
    cudaError_t e = cudaMemcpyAsync(y, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, h->stream);
    return e == cudaSuccess ? LB_OK : cuda_fail(h, e, "copy");
}

int k_scale_rows(Handle* h, double* z, const double* v, const double* coef, int nm, size_t NENK) {
    if (nm < 1 || nm > kMaxRowCoefs) return fail(h, LB_ERR_ARG, "k_scale_rows: too many moment rows");
    RowCoefs rc{};
    for (int j = 0; j < nm; ++j) rc.c[j] = coef[j];
    Timer t;
    timer_begin(h, LB_T_PRECOND, t);
    int gx = grid_for(h, NENK * (size_t)nm) / nm;
    dim3 grid(gx < 1 ? 1 : gx, nm);
    scale_rows_kernel<<<grid, 256, 0, h->stream>>>(z, v, rc, NENK);
    timer_end(h, t);
    return LB_OK;
}

int k_fill(Handle* h, double* y, double v, size_t n) {
    Timer t;
    timer_begin(h, LB_T_KRYLOV, t);
    fill_kernel<<<grid_for(h, n), 256, 0, h->stream>>>(y, v, n);
    timer_end(h, t);
    return LB_OK;
}

int k_f64_to_f32(Handle* h, float* y, const double* x, size_t n) {
    Timer t;
    timer_begin(h, LB_T_COPY, t);
    f64_to_f32_kernel<<<grid_for(h, n), 256, 0, h->stream>>>(y, x, n);
    timer_end(h, t);
    return LB_OK;
}

int k_f32_to_f64(Handle* h, double* y, const float* x, size_t n) {
    Timer t;
    timer_begin(h, LB_T_COPY, t);
    f32_to_f64_kernel<<<grid_for(h, n), 256, 0, h->stream>>>(y, x, n);
    timer_end(h, t);
    return LB_OK;
}

int k_moment_source(Handle* h, double* src, const double* phi, const float* sigl, const int* mat, long long NENK, int nm,
                    int nmpad, int accumulate) {
    Timer t;
    timer_begin(h, LB_T_TALLY, t);
    moment_source_kernel<<<grid_for(h, (size_t)nm * NENK), 256, 0, h->stream>>>(src, phi, sigl, mat, NENK, nm, nmpad, accumulate);
    timer_end(h, t);
    return LB_OK;
}

int k_unc_source(Handle* h, double* src, const double* unc, const double* ybeam, const float* sigl, const int* mat,
                 long long NENK, int nm, int nmpad) {
    Timer t;
    timer_begin(h, LB_T_TALLY, t);
    unc_source_kernel<<<grid_for(h, (size_t)nm * NENK), 256, 0, h->stream>>>(src, unc, ybeam, sigl, mat, NENK, nm, nmpad);
    timer_end(h, t);
    return LB_OK;
}

int k_group_source(Handle* h, double* src, const double* phi_all, const float* tab, int G, int g, const double* unc,
                   const double* ybeam, const int* mat, long long NENK, int Nm, int nm, int nmpad) {
    Timer t;
    timer_begin(h, LB_T_TALLY, t);
    group_source_kernel<<<grid_for(h, (size_t)NENK / 4), 256, 0, h->stream>>>(src, phi_all, tab, G, g, unc, ybeam, mat, NENK,
                                                                           Nm, nm, nmpad);
    timer_end(h, t);
    return LB_OK;
}

int k_dose_tally(Handle* h, const double* phi00, const double* unc, double unc_scale, const double* dd_mat, const int* mat,
                 double* flux, double* dose, long long NENK) {
    Timer t;
    timer_begin(h, LB_T_TALLY, t);
    dose_kernel<<<grid_for(h, (size_t)NENK), 256, 0, h->stream>>>(phi00, unc, unc_scale, dd_mat, mat, flux, dose, NENK);
    timer_end(h, t);
    return LB_OK;
}


// ---------------------------------------------------------------------------------------------
//  segmented operations of a batch
// ---------------------------------------------------------------------------------------------
int seg_assign_blocks(std::vector<SegVec>& segs, int blocks) {
    double tot = 0.0;
    for (auto& sg : segs) tot += (double)sg.n2;
    int b0 = 0;
    for (auto& sg : segs) {
        int nb = (int)std::floor((double)blocks * (double)sg.n2 / std::max(tot, 1.0));
        nb = std::max(nb, 1);
        sg.blk0 = b0;
        sg.nblk = nb;
        b0 += nb;
    }
    return b0;
}

// Uploads the segment table (and coefficients) through the handle's pinned staging area.
static int seg_upload(Handle* h, const std::vector<SegVec>& segs, const std::vector<double>* coef, SegVec** dsegs,
                      double** dcoef) {
    const size_t sb = sizeof(SegVec) * segs.size();
    const size_t cb = coef ? sizeof(double) * coef->size() : 0;
    const size_t need = sb + cb + 64;
    if (need > h->seg_bytes) {
        if (h->d_seg) cudaFree(h->d_seg);
        if (h->h_seg) cudaFreeHost(h->h_seg);
        h->d_seg = nullptr;
        h->h_seg = nullptr;
        h->seg_bytes = 0;
        const size_t cap = std::max<size_t>(need * 2, 1 << 16);
        if (cudaMalloc(&h->d_seg, cap) != cudaSuccess || cudaMallocHost(&h->h_seg, cap) != cudaSuccess)
            return fail(h, LB_ERR_OOM, "segment tables");
        h->seg_bytes = cap;
    }
    // the staging buffer is reused by the next call: wait for the previous upload to be consumed
    cudaStreamSynchronize(h->stream);
    unsigned char* hb = reinterpret_cast<unsigned char*>(h->h_seg);
    std::memcpy(hb, segs.data(), sb);
    const size_t coff = (sb + 15) / 16 * 16;
    if (cb) std::memcpy(hb + coff, coef->data(), cb);
    cudaError_t e = cudaMemcpyAsync(h->d_seg, hb, coff + cb, cudaMemcpyHostToDevice, h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "segment upload");
    *dsegs = reinterpret_cast<SegVec*>(h->d_seg);
    if (dcoef) *dcoef = reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(h->d_seg) + coff);
    return LB_OK;
}

static int seg_reduce(Handle* h, const std::vector<SegVec>& segs, int cnt, std::vector<double>& out) {
    const int grid = segs.back().blk0 + segs.back().nblk;
    cudaError_t e = cudaMemcpyAsync(h->h_red, h->d_red, sizeof(double) * (size_t)grid * kPartStride,
                                    cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "segmented reduction");
    out.assign(segs.size() * (size_t)cnt, 0.0);
    for (size_t si = 0; si < segs.size(); ++si)
        for (int j = 0; j < cnt; ++j) {
            double acc = 0.0;
            for (int b = segs[si].blk0; b < segs[si].blk0 + segs[si].nblk; ++b) acc += h->h_red[(size_t)b * kPartStride + j];
            out[si * cnt + j] = acc;
        }
    return LB_OK;
}

int seg_dots_norm(Handle* h, const std::vector<SegVec>& segs, int nv, std::vector<double>& out) {
    if (segs.empty()) { out.clear(); return LB_OK; }
    if (nv < 0 || nv > kMaxDots) return fail(h, LB_ERR_ARG, "segmented dots: too many vectors");
    SegVec* ds = nullptr;
    int rc = seg_upload(h, segs, nullptr, &ds, nullptr);
    if (rc) return rc;
    const int grid = segs.back().blk0 + segs.back().nblk;
    NvDispatch<kMaxDots>::run(nv, [&](auto c) {
        constexpr int NV = decltype(c)::value;
        seg_dots_t<NV><<<grid, kRedThreads, 0, h->stream>>>(ds, (int)segs.size(), h->d_red);
    });
    return seg_reduce(h, segs, nv + 1, out);
}

int seg_axpy_dots(Handle* h, const std::vector<SegVec>& segs, int nv, const std::vector<double>& coef, bool dots,
                  std::vector<double>& out) {
    if (segs.empty()) { out.clear(); return LB_OK; }
    if (nv < 0 || nv > kMaxDots) return fail(h, LB_ERR_ARG, "segmented axpy: too many vectors");
    SegVec* ds = nullptr;
    double* dc = nullptr;
    int rc = seg_upload(h, segs, &coef, &ds, &dc);
    if (rc) return rc;
    const int grid = segs.back().blk0 + segs.back().nblk;
    NvDispatch<kMaxDots>::run(nv, [&](auto c) {
        constexpr int NV = decltype(c)::value;
        if (dots) seg_axpy_dots_t<NV, true><<<grid, kRedThreads, 0, h->stream>>>(ds, (int)segs.size(), dc, h->d_red);
        else seg_axpy_dots_t<NV, false><<<grid, kRedThreads, 0, h->stream>>>(ds, (int)segs.size(), dc, h->d_red);
    });
    return seg_reduce(h, segs, nv + 1, out);
}

int seg_axpy_scale(Handle* h, const std::vector<SegVec>& segs, int nv, const std::vector<double>& coef) {
    if (segs.empty()) return LB_OK;
    if (nv < 0 || nv > kMaxDots) return fail(h, LB_ERR_ARG, "segmented axpy: too many vectors");
    SegVec* ds = nullptr;
    double* dc = nullptr;
    int rc = seg_upload(h, segs, &coef, &ds, &dc);
    if (rc) return rc;
    const int grid = segs.back().blk0 + segs.back().nblk;
    NvDispatch<kMaxDots>::run(nv, [&](auto c) {
        constexpr int NV = decltype(c)::value;
        seg_axpy_scale_t<NV><<<grid, kRedThreads, 0, h->stream>>>(ds, (int)segs.size(), dc);
    });
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LB_OK : cuda_fail(h, e, "segmented axpy");
}

int seg_axpby_norm(Handle* h, const std::vector<SegVec>& segs, std::vector<double>& out) {
    if (segs.empty()) { out.clear(); return LB_OK; }
    SegVec* ds = nullptr;
    int rc = seg_upload(h, segs, nullptr, &ds, nullptr);
    if (rc) return rc;
    const int grid = segs.back().blk0 + segs.back().nblk;
    seg_axpby_norm_kernel<<<grid, kRedThreads, 0, h->stream>>>(ds, (int)segs.size(), h->d_red);
    return seg_reduce(h, segs, 1, out);
}

}  // namespace lb
