// FP64 vector kernels for the flux-moment Krylov solvers (GMRES/FGMRES/SI) and the multigroup
// source / dose tallies.  The reference runs these as serial Fortran loops inside SPARSKIT
// (third_party/SPARSKIT/iters.f: gmres :1901-2206, mgsro :3465-3587) and Main.f90.
// Reductions are deterministic: fixed grid, per-block partials summed on the host in block order.
#include "lb_internal.h"

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

// partial[b][j] = sum over this block's share of q of V[j][q] * w[q], j < nv.
// Vectors are read as double2 (n is even: n = nm * NENK with NENK a multiple of 4).
__global__ void __launch_bounds__(kRedThreads) dots_kernel(const double* __restrict__ V, size_t ldv, int nv,
                                                          const double* __restrict__ w, size_t n, double* partial) {
    __shared__ double s[kRedThreads / 32][kMaxDots];
    double acc[kMaxDots];
#pragma unroll
    for (int j = 0; j < kMaxDots; ++j) acc[j] = 0.0;
    const size_t n2 = n / 2;
    const double2* w2 = reinterpret_cast<const double2*>(w);
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n2; q += (size_t)gridDim.x * blockDim.x) {
        const double2 wq = __ldcs(&w2[q]);
#pragma unroll
        for (int j = 0; j < kMaxDots; ++j)
            if (j < nv) {
                const double2 v = __ldcs(reinterpret_cast<const double2*>(V + (size_t)j * ldv) + q);
                acc[j] = fma(v.x, wq.x, fma(v.y, wq.y, acc[j]));
            }
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int j = 0; j < kMaxDots; ++j) {
        if (j < nv) {
            double v = warp_sum(acc[j]);
            if (lane == 0) s[warp][j] = v;
        }
    }
    __syncthreads();
    if (threadIdx.x < nv) {
        double v = 0.0;
        for (int k = 0; k < kRedThreads / 32; ++k) v += s[k][threadIdx.x];
        partial[(size_t)blockIdx.x * kMaxDots + threadIdx.x] = v;
    }
}

// w -= sum_j c[j] V[j];  partial[b] = sum of w^2 over the block (after the update)
__global__ void __launch_bounds__(kRedThreads) axpy_norm_kernel(double* w, const double* __restrict__ V, size_t ldv, int nv,
                                                               Coefs cf, size_t n, double* partial) {
    __shared__ double s[kRedThreads / 32];
    double acc = 0.0;
    const size_t n2 = n / 2;
    double2* w2 = reinterpret_cast<double2*>(w);
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n2; q += (size_t)gridDim.x * blockDim.x) {
        double2 v = w2[q];
#pragma unroll
        for (int j = 0; j < kMaxDots; ++j)
            if (j < nv) {
                const double2 u = __ldcs(reinterpret_cast<const double2*>(V + (size_t)j * ldv) + q);
                v.x = fma(-cf.c[j], u.x, v.x);
                v.y = fma(-cf.c[j], u.y, v.y);
            }
        w2[q] = v;
        acc = fma(v.x, v.x, fma(v.y, v.y, acc));
    }
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = 0.0;
        for (int k = 0; k < kRedThreads / 32; ++k) v += s[k];
        partial[blockIdx.x] = v;
    }
}

__global__ void axpby_kernel(double* y, const double* x, double a, double b, size_t n) {
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
        y[q] = a * x[q] + b * y[q];
}

__global__ void scale_kernel(double* y, double a, size_t n) {
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) y[q] *= a;
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

inline int grid_for(Handle* h, size_t n) {
    size_t g = (n + 255) / 256;
    size_t cap = (size_t)h->sm_count * 8;
    return (int)std::max<size_t>(1, std::min(g, cap));
}

}  // namespace

int k_dots(Handle* h, const double* V, size_t ldv, int nv, const double* w, size_t n, double* out) {
    if (nv > kMaxDots) return fail(h, LB_ERR_ARG, "dots: too many vectors");
    if (n % 2) return fail(h, LB_ERR_ARG, "dots: odd vector length");
    const int grid = h->sm_count * 4;
    Timer t;
    timer_begin(h, LB_T_KRYLOV, t);
    dots_kernel<<<grid, kRedThreads, 0, h->stream>>>(V, ldv, nv, w, n, h->d_red);
    timer_end(h, t);
    cudaError_t e = cudaMemcpyAsync(h->h_red, h->d_red, sizeof(double) * grid * kMaxDots, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "dots");
    for (int j = 0; j < nv; ++j) {
        double s = 0.0;
        for (int b = 0; b < grid; ++b) s += h->h_red[(size_t)b * kMaxDots + j];
        out[j] = s;
    }
    return LB_OK;
}

// w -= sum_j coef[j] V[j]; returns ||w||^2 through *nrm2 (may be null)
int k_multi_axpy_norm(Handle* h, double* w, const double* V, size_t ldv, int nv, const double* coef, size_t n, double* nrm2) {
    if (nv > kMaxDots) return fail(h, LB_ERR_ARG, "axpy: too many vectors");
    if (n % 2) return fail(h, LB_ERR_ARG, "axpy: odd vector length");
    Coefs cf;
    for (int j = 0; j < kMaxDots; ++j) cf.c[j] = (j < nv) ? coef[j] : 0.0;
    const int grid = h->sm_count * 4;
    Timer t;
    timer_begin(h, LB_T_KRYLOV, t);
    axpy_norm_kernel<<<grid, kRedThreads, 0, h->stream>>>(w, V, ldv, nv, cf, n, h->d_red);
    timer_end(h, t);
    if (!nrm2) return LB_OK;
    cudaError_t e = cudaMemcpyAsync(h->h_red, h->d_red, sizeof(double) * grid, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "axpy_norm");
    double s = 0.0;
    for (int b = 0; b < grid; ++b) s += h->h_red[b];
    *nrm2 = s;
    return LB_OK;
}

int k_multi_axpy(Handle* h, double* w, const double* V, size_t ldv, int nv, const double* coef, size_t n) {
    return k_multi_axpy_norm(h, w, V, ldv, nv, coef, n, nullptr);
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

int k_dose_tally(Handle* h, const double* phi00, const double* unc, double unc_scale, const double* dd_mat, const int* mat,
                 double* flux, double* dose, long long NENK) {
    Timer t;
    timer_begin(h, LB_T_TALLY, t);
    dose_kernel<<<grid_for(h, (size_t)NENK), 256, 0, h->stream>>>(phi00, unc, unc_scale, dd_mat, mat, flux, dose, NENK);
    timer_end(h, t);
    return LB_OK;
}

}  // namespace lb
