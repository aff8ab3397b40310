// Scattering as two dense moment contractions on the tensor cores, sm_100a.
//
// The reference applies K as a dense NI x NI discrete-to-discrete kernel,
//   (Kx)(i) = sum_i' YYS(i',i) x(i'),  YYS = sum_l XS%s(l) w(i') (2l+1)/(4pi) P_l(k_i.k_i')
// (ScatteringOperator.f90:263-269, ScatteringAlgebra.f90:13-55).  By the addition theorem
// P_l(a.b) (2l+1)/(4pi) = sum_m Y_lm(a) Y_lm(b) this factorises exactly into
//   D2M: phi_j(n) = sum_i w_i Y_j(k_i) psi_i(n)           [nm x NI] . [NI x NENK]
//   M2D: q_i(n)   = sum_j Y_j(k_i) sigma_l(j)(mat(n)) phi_j(n)
// Both run as mma.sync m16n8k16 BF16 products with FP32 accumulation.  Each FP32 operand value
// is split into three BF16 planes (hi + mid + lo = 24 significant bits) and the six products
// whose magnitude exceeds 2^-24 of the leading term are accumulated (hi.hi, hi.mid, mid.hi,
// hi.lo, mid.mid, lo.hi), which reproduces an FP32 GEMM on the BF16 tensor pipe.
#include "lb_internal.h"
#include <cstdlib>

namespace lb {

namespace {

constexpr int kTileN = 64;      // nodes per CTA tile
constexpr int kThreads = 256;   // 8 warps; warp w owns n8 tile w of the CTA tile

__device__ __forceinline__ void split3(float v, __nv_bfloat16& a, __nv_bfloat16& b, __nv_bfloat16& c) {
    a = __float2bfloat16_rn(v);
    float r1 = v - __bfloat162float(a);
    b = __float2bfloat16_rn(r1);
    float r2 = r1 - __bfloat162float(b);
    c = __float2bfloat16_rn(r2);
}

__device__ __forceinline__ void mma16816(float* d, const uint32_t* a, const uint32_t* b) {
    asm(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// The six split products, small terms first.
__device__ __forceinline__ void mma_split6(float* d, const uint32_t (*a)[4], const uint32_t (*b)[2]) {
    mma16816(d, a[2], b[0]);   // lo.hi
    mma16816(d, a[1], b[1]);   // mid.mid
    mma16816(d, a[0], b[2]);   // hi.lo
    mma16816(d, a[1], b[0]);   // mid.hi
    mma16816(d, a[0], b[1]);   // hi.mid
    mma16816(d, a[0], b[0]);   // hi.hi
}

// row stride (32-bit words) of a [n][k] BF16 smem operand: == 4 mod 8 so that the 8 rows read
// by one fragment load land in distinct banks
__host__ __device__ __forceinline__ int smem_stride_words(int kpad) {
    int s = kpad / 2;
    return s + ((4 - (s % 8)) + 8) % 8;
}

// ---------------------------------------------------------------------------------------------
// M2D: q[i][n] = sum_j Y[i][j] * xt[j][n] (+ qadd[i][n]),
//      xt[j][n] = sigl[mat(n)][j] * x[j][n] + a[j][n]
// A = Y planes [3][NIpad][nmpad] (global, L1-resident), B = xt tile in smem as [3][n][j].
// Warp w computes all direction tiles for the 8 nodes of n8 tile w.
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) m2d_kernel(const int* __restrict__ active, const double* __restrict__ x, const float* __restrict__ sigl,
                                                      const double* __restrict__ add, const float* __restrict__ qadd,
                                                      const int* __restrict__ mat, const __nv_bfloat16* __restrict__ Y,
                                                      float* __restrict__ q, long long NENK, int NI, int NIpad,
                                                      int nm, int nmpad, long long ntiles) {
    if (active && *active == 0) return;   // problem of a batch that has converged
    extern __shared__ __align__(16) uint32_t smem[];
    const int sw = smem_stride_words(nmpad);            // words per node row
    uint32_t* Bs = smem;                                  // [3][kTileN][sw]
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = lane >> 2, t = lane & 3;
    const size_t plane = (size_t)NIpad * nmpad;
    const uint32_t* Yw = reinterpret_cast<const uint32_t*>(Y);
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long long n0 = tile * kTileN;
        __syncthreads();
        // prepass: scale, split, transpose into smem
        for (int idx = tid; idx < kTileN * nmpad; idx += kThreads) {
            const int j = idx / kTileN, nn = idx % kTileN;
            const long long n = n0 + nn;
            float v = 0.f;
            if (j < nm && n < NENK) {
                double s = 0.0;
                if (x) s = (double)__ldg(&sigl[(size_t)__ldg(&mat[n >> 2]) * nmpad + j]) * x[(size_t)j * NENK + n];
                if (add) s += add[(size_t)j * NENK + n];
                v = (float)s;
            }
            __nv_bfloat16 a, b, c;
            split3(v, a, b, c);
            __nv_bfloat16* row0 = reinterpret_cast<__nv_bfloat16*>(Bs + (size_t)(0 * kTileN + nn) * sw);
            __nv_bfloat16* row1 = reinterpret_cast<__nv_bfloat16*>(Bs + (size_t)(1 * kTileN + nn) * sw);
            __nv_bfloat16* row2 = reinterpret_cast<__nv_bfloat16*>(Bs + (size_t)(2 * kTileN + nn) * sw);
            row0[j] = a; row1[j] = b; row2[j] = c;
        }
        __syncthreads();
        const int nb = warp * 8;       // this warp's n8 tile inside the CTA tile
        for (int m0 = 0; m0 < NIpad; m0 += 16) {
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
            for (int k0 = 0; k0 < nmpad; k0 += 16) {
                uint32_t af[3][4], bf[3][2];
#pragma unroll
                for (int p = 0; p < 3; ++p) {
                    const uint32_t* Yp = Yw + (p * plane) / 2;
                    af[p][0] = __ldg(&Yp[((size_t)(m0 + g) * nmpad + k0 + 2 * t) / 2]);
                    af[p][1] = __ldg(&Yp[((size_t)(m0 + g + 8) * nmpad + k0 + 2 * t) / 2]);
                    af[p][2] = __ldg(&Yp[((size_t)(m0 + g) * nmpad + k0 + 2 * t + 8) / 2]);
                    af[p][3] = __ldg(&Yp[((size_t)(m0 + g + 8) * nmpad + k0 + 2 * t + 8) / 2]);
                    const uint32_t* Bp = Bs + (size_t)(p * kTileN + nb + g) * sw;
                    bf[p][0] = Bp[(k0 + 2 * t) / 2];
                    bf[p][1] = Bp[(k0 + 2 * t + 8) / 2];
                }
                mma_split6(acc, af, bf);
            }
            // epilogue: rows m0+g, m0+g+8; nodes nb + 2t, +1
            const long long n = n0 + nb + 2 * t;
            if (n < NENK) {
                const int r0 = m0 + g, r1 = m0 + g + 8;
                if (r0 < NI) {
                    float2 v = make_float2(acc[0], acc[1]);
                    if (qadd) { float2 u = *reinterpret_cast<const float2*>(&qadd[(size_t)r0 * NENK + n]); v.x += u.x; v.y += u.y; }
                    __stcs(reinterpret_cast<float2*>(&q[(size_t)r0 * NENK + n]), v);
                }
                if (r1 < NI) {
                    float2 v = make_float2(acc[2], acc[3]);
                    if (qadd) { float2 u = *reinterpret_cast<const float2*>(&qadd[(size_t)r1 * NENK + n]); v.x += u.x; v.y += u.y; }
                    __stcs(reinterpret_cast<float2*>(&q[(size_t)r1 * NENK + n]), v);
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------------------------
// D2M: z[j][n] = sum_i Dw[j][i] psi[i][n];  out[j][n] = alpha * xin[j][n] + beta * z[j][n]
// A = Dw planes [3][nmpad][NIpad] (global), B = psi tile split into smem as [3][n][i].
// ---------------------------------------------------------------------------------------------
template <int MT>
__global__ void __launch_bounds__(kThreads) d2m_kernel(const int* __restrict__ active, const float* __restrict__ psi, const __nv_bfloat16* __restrict__ Dw,
                                                      const double* __restrict__ xin, double alpha, double beta,
                                                      double* __restrict__ out, long long NENK, int NI, int NIpad,
                                                      int nm, int nmpad, long long ntiles) {
    if (active && *active == 0) return;   // problem of a batch that has converged
    extern __shared__ __align__(16) uint32_t smem[];
    const int sw = smem_stride_words(NIpad);
    uint32_t* Bs = smem;                                  // [3][kTileN][sw]
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = lane >> 2, t = lane & 3;
    const size_t plane = (size_t)nmpad * NIpad;
    const uint32_t* Dwd = reinterpret_cast<const uint32_t*>(Dw);
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long long n0 = tile * kTileN;
        __syncthreads();
        // prepass: psi rows are read as float4 along the nodes, split, transposed into smem
        for (int idx = tid; idx < NIpad * (kTileN / 4); idx += kThreads) {
            const int i = idx / (kTileN / 4), q4 = idx % (kTileN / 4);
            const long long n = n0 + 4 * q4;
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (i < NI && n < NENK) v = __ldcs(reinterpret_cast<const float4*>(&psi[(size_t)i * NENK + n]));
            const float vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                __nv_bfloat16 a, b, d;
                split3(vv[c], a, b, d);
                const int nn = 4 * q4 + c;
                reinterpret_cast<__nv_bfloat16*>(Bs + (size_t)(0 * kTileN + nn) * sw)[i] = a;
                reinterpret_cast<__nv_bfloat16*>(Bs + (size_t)(1 * kTileN + nn) * sw)[i] = b;
                reinterpret_cast<__nv_bfloat16*>(Bs + (size_t)(2 * kTileN + nn) * sw)[i] = d;
            }
        }
        __syncthreads();
        const int nb = warp * 8;
        float acc[MT][4];
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) acc[mt][0] = acc[mt][1] = acc[mt][2] = acc[mt][3] = 0.f;
        const int mtiles = nmpad / 16;
        for (int k0 = 0; k0 < NIpad; k0 += 16) {
            uint32_t bf[3][2];
#pragma unroll
            for (int p = 0; p < 3; ++p) {
                const uint32_t* Bp = Bs + (size_t)(p * kTileN + nb + g) * sw;
                bf[p][0] = Bp[(k0 + 2 * t) / 2];
                bf[p][1] = Bp[(k0 + 2 * t + 8) / 2];
            }
#pragma unroll
            for (int mt = 0; mt < MT; ++mt) {
                if (mt >= mtiles) break;
                const int m0 = mt * 16;
                uint32_t af[3][4];
#pragma unroll
                for (int p = 0; p < 3; ++p) {
                    const uint32_t* Dp = Dwd + (p * plane) / 2;
                    af[p][0] = __ldg(&Dp[((size_t)(m0 + g) * NIpad + k0 + 2 * t) / 2]);
                    af[p][1] = __ldg(&Dp[((size_t)(m0 + g + 8) * NIpad + k0 + 2 * t) / 2]);
                    af[p][2] = __ldg(&Dp[((size_t)(m0 + g) * NIpad + k0 + 2 * t + 8) / 2]);
                    af[p][3] = __ldg(&Dp[((size_t)(m0 + g + 8) * NIpad + k0 + 2 * t + 8) / 2]);
                }
                mma_split6(acc[mt], af, bf);
            }
        }
        const long long n = n0 + nb + 2 * t;
        if (n < NENK) {
#pragma unroll
            for (int mt = 0; mt < MT; ++mt) {
                if (mt >= mtiles) break;
                const int r0 = mt * 16 + g, r1 = r0 + 8;
                if (r0 < nm) {
                    double2 v = make_double2(beta * (double)acc[mt][0], beta * (double)acc[mt][1]);
                    if (xin) { double2 u = *reinterpret_cast<const double2*>(&xin[(size_t)r0 * NENK + n]); v.x += alpha * u.x; v.y += alpha * u.y; }
                    *reinterpret_cast<double2*>(&out[(size_t)r0 * NENK + n]) = v;
                }
                if (r1 < nm) {
                    double2 v = make_double2(beta * (double)acc[mt][2], beta * (double)acc[mt][3]);
                    if (xin) { double2 u = *reinterpret_cast<const double2*>(&xin[(size_t)r1 * NENK + n]); v.x += alpha * u.x; v.y += alpha * u.y; }
                    *reinterpret_cast<double2*>(&out[(size_t)r1 * NENK + n]) = v;
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Streaming versions.  The constant operand (Y or w*Y planes) is copied once per persistent CTA into
// shared memory with rows padded to an odd multiple of 16 bytes and fed to the tensor cores with
// ldmatrix; the data operand streams from HBM straight into mma fragments (each warp load instruction
// touches 4 rows x 32 contiguous bytes) and is split into BF16 planes in registers.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ void ldsm_x4(uint32_t* r, const void* smem_row) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(smem_row);
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(a));
}

// (v0, v1) -> packed hi / mid / lo BF16 pairs (low half = v0)
__device__ __forceinline__ void split_pair(float v0, float v1, uint32_t& hi, uint32_t& mid, uint32_t& lo) {
    __nv_bfloat162 h = __floats2bfloat162_rn(v0, v1);
    float2 fh = __bfloat1622float2(h);
    const float r0 = v0 - fh.x, r1 = v1 - fh.y;
    __nv_bfloat162 m = __floats2bfloat162_rn(r0, r1);
    float2 fm = __bfloat1622float2(m);
    __nv_bfloat162 l = __floats2bfloat162_rn(r0 - fm.x, r1 - fm.y);
    hi = *reinterpret_cast<uint32_t*>(&h);
    mid = *reinterpret_cast<uint32_t*>(&m);
    lo = *reinterpret_cast<uint32_t*>(&l);
}

// Copy the [3][rows][cols] BF16 planes into shared memory with row stride cols + 8.
__device__ __forceinline__ void stage_planes(const __nv_bfloat16* __restrict__ g, __nv_bfloat16* s, int rows, int cols) {
    const int cw = cols / 8, rs = cols + 8;      // 16-byte chunks per row, padded row stride (halves)
    const int total = 3 * rows * cw;
    for (int c = threadIdx.x; c < total; c += blockDim.x) {
        const int pr = c / cw, q = c % cw;       // pr = plane*rows + row
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(g + (size_t)pr * cols) + q);
        *reinterpret_cast<uint4*>(s + (size_t)pr * rs + q * 8) = v;
    }
    __syncthreads();
}

// M2D: q[i][n] = sum_j Y[i][j] xt[j][n] (+ qadd),  xt = sigl[mat(n)][j] x[j][n] + a[j][n].
// NW warps per CTA; warp w owns nodes n0 + 8w .. +7 of the 8*NW-node tile; its B fragments for all
// K stay in registers.  Direction tiles are processed in pairs: two independent accumulator chains.
template <int KT, int NW>
__global__ void __launch_bounds__(NW * 32, 1) m2d_stream_kernel(const int* __restrict__ active, const double* __restrict__ x, const float* __restrict__ sigl,
                                                             const double* __restrict__ add, const float* __restrict__ qadd,
                                                             const int* __restrict__ mat, const __nv_bfloat16* __restrict__ Y,
                                                             float* __restrict__ q, long long NENK, int NI, int NIpad,
                                                             int nm, int nmpad, long long ntiles) {
    if (active && *active == 0) return;   // problem of a batch that has converged
    extern __shared__ __align__(16) __nv_bfloat16 ys[];     // [3][NIpad][nmpad + 8]
    stage_planes(Y, ys, NIpad, nmpad);
    constexpr int TN = NW * 8;
    const int rs = nmpad + 8;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const int mi = lane >> 3, rr = lane & 7;                // ldmatrix: matrix index, row in matrix
    const int arow = rr + 8 * (mi & 1), acol = 8 * (mi >> 1);
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long long n = tile * TN + warp * 8 + g;       // node of this thread's B column
        const bool nok = n < NENK;
        const int m = nok ? __ldg(&mat[n >> 2]) : 0;
        uint32_t bf[KT][3][2];
#pragma unroll
        for (int kt = 0; kt < KT; ++kt) {
            float v[4];
#pragma unroll
            for (int h = 0; h < 4; ++h) {
                const int j = kt * 16 + 2 * t + (h & 1) + 8 * (h >> 1);
                double s = 0.0;
                if (nok && j < nm) {
                    if (x) s = (double)__ldg(&sigl[(size_t)m * nmpad + j]) * __ldcs(&x[(size_t)j * NENK + n]);
                    if (add) s += __ldcs(&add[(size_t)j * NENK + n]);
                }
                v[h] = (float)s;
            }
            split_pair(v[0], v[1], bf[kt][0][0], bf[kt][1][0], bf[kt][2][0]);
            split_pair(v[2], v[3], bf[kt][0][1], bf[kt][1][1], bf[kt][2][1]);
        }
        const long long nc = tile * TN + warp * 8 + 2 * t;   // output column pair of this thread
        auto store = [&](int m0, const float* acc) {
            if (nc >= NENK) return;
            const int r0 = m0 + g, r1 = m0 + g + 8;
            if (r0 < NI) {
                float2 v = make_float2(acc[0], acc[1]);
                if (qadd) { float2 u = *reinterpret_cast<const float2*>(&qadd[(size_t)r0 * NENK + nc]); v.x += u.x; v.y += u.y; }
                __stcs(reinterpret_cast<float2*>(&q[(size_t)r0 * NENK + nc]), v);
            }
            if (r1 < NI) {
                float2 v = make_float2(acc[2], acc[3]);
                if (qadd) { float2 u = *reinterpret_cast<const float2*>(&qadd[(size_t)r1 * NENK + nc]); v.x += u.x; v.y += u.y; }
                __stcs(reinterpret_cast<float2*>(&q[(size_t)r1 * NENK + nc]), v);
            }
        };
        int m0 = 0;
        for (; m0 + 16 < NIpad; m0 += 32) {
            float acc0[4] = {0.f, 0.f, 0.f, 0.f}, acc1[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int kt = 0; kt < KT; ++kt) {
                uint32_t a0[3][4], a1[3][4];
#pragma unroll
                for (int p = 0; p < 3; ++p) {
                    ldsm_x4(a0[p], ys + ((size_t)p * NIpad + m0 + arow) * rs + kt * 16 + acol);
                    ldsm_x4(a1[p], ys + ((size_t)p * NIpad + m0 + 16 + arow) * rs + kt * 16 + acol);
                }
                mma_split6(acc0, a0, bf[kt]);
                mma_split6(acc1, a1, bf[kt]);
            }
            store(m0, acc0);
            store(m0 + 16, acc1);
        }
        if (m0 < NIpad) {
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int kt = 0; kt < KT; ++kt) {
                uint32_t af[3][4];
#pragma unroll
                for (int p = 0; p < 3; ++p)
                    ldsm_x4(af[p], ys + ((size_t)p * NIpad + m0 + arow) * rs + kt * 16 + acol);
                mma_split6(acc, af, bf[kt]);
            }
            store(m0, acc);
        }
    }
}

// D2M: z[j][n] = sum_i Dw[j][i] psi[i][n];  out = alpha * xin + beta * z.
// NW warps per CTA; warp w owns nodes n0 + 8w .. +7; psi fragments stream from HBM one k-step ahead
// of the MMAs.
template <int MT, int NW>
__global__ void __launch_bounds__(NW * 32, 1) d2m_stream_kernel(const int* __restrict__ active, const float* __restrict__ psi, const __nv_bfloat16* __restrict__ Dw,
                                                             const double* xin, double alpha, double beta, double* out,
                                                             long long NENK, int NI, int NIpad, int nm, int nmpad,
                                                             long long ntiles) {
    if (active && *active == 0) return;   // problem of a batch that has converged
    extern __shared__ __align__(16) __nv_bfloat16 ds[];     // [3][nmpad][NIpad + 8]
    stage_planes(Dw, ds, nmpad, NIpad);
    const int rs = NIpad + 8;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const int mi = lane >> 3, rr = lane & 7;
    const int arow = rr + 8 * (mi & 1), acol = 8 * (mi >> 1);
    const int mtiles = nmpad / 16;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long long n = tile * (NW * 8) + warp * 8 + g;
        const bool nok = n < NENK;
        float acc[MT][4];
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) acc[mt][0] = acc[mt][1] = acc[mt][2] = acc[mt][3] = 0.f;
        auto load = [&](int k0, float* v) {
#pragma unroll
            for (int h = 0; h < 4; ++h) {
                const int i = k0 + 2 * t + (h & 1) + 8 * (h >> 1);
                v[h] = (nok && i < NI) ? __ldcs(&psi[(size_t)i * NENK + n]) : 0.f;
            }
        };
        float cur[4], nxt[4];
        load(0, cur);
        for (int k0 = 0; k0 < NIpad; k0 += 16) {
            if (k0 + 16 < NIpad) load(k0 + 16, nxt);
            uint32_t bf[3][2];
            split_pair(cur[0], cur[1], bf[0][0], bf[1][0], bf[2][0]);
            split_pair(cur[2], cur[3], bf[0][1], bf[1][1], bf[2][1]);
#pragma unroll
            for (int mt = 0; mt < MT; ++mt) {
                if (mt >= mtiles) break;
                uint32_t af[3][4];
#pragma unroll
                for (int p = 0; p < 3; ++p)
                    ldsm_x4(af[p], ds + ((size_t)p * nmpad + mt * 16 + arow) * rs + k0 + acol);
                mma_split6(acc[mt], af, bf);
            }
#pragma unroll
            for (int h = 0; h < 4; ++h) cur[h] = nxt[h];
        }
        const long long nc = tile * (NW * 8) + warp * 8 + 2 * t;
        if (nc < NENK) {
#pragma unroll
            for (int mt = 0; mt < MT; ++mt) {
                if (mt >= mtiles) break;
                const int r0 = mt * 16 + g, r1 = r0 + 8;
                if (r0 < nm) {
                    double2 v = make_double2(beta * (double)acc[mt][0], beta * (double)acc[mt][1]);
                    if (xin) { double2 u = *reinterpret_cast<const double2*>(&xin[(size_t)r0 * NENK + nc]); v.x += alpha * u.x; v.y += alpha * u.y; }
                    *reinterpret_cast<double2*>(&out[(size_t)r0 * NENK + nc]) = v;
                }
                if (r1 < nm) {
                    double2 v = make_double2(beta * (double)acc[mt][2], beta * (double)acc[mt][3]);
                    if (xin) { double2 u = *reinterpret_cast<const double2*>(&xin[(size_t)r1 * NENK + nc]); v.x += alpha * u.x; v.y += alpha * u.y; }
                    *reinterpret_cast<double2*>(&out[(size_t)r1 * NENK + nc]) = v;
                }
            }
        }
    }
}

template <int MT>
int run_d2m(Handle* h, const float* psi, const double* xin, double alpha, double beta, double* out, long long ntiles,
            int grid, size_t smem) {
    static PerDevice attr;
    attr.get([&] {
        allow_max_dynamic_smem(d2m_kernel<MT>);
        return 1;
    });
    d2m_kernel<MT><<<grid, kThreads, smem, h->stream>>>(h->d_active, psi, h->d_Yd2m, xin, alpha, beta, out, h->NENK, h->NI,
                                                        h->NIpad, h->nm, h->nmpad, ntiles);
    return LB_OK;
}


template <int KT, int NW>
cudaError_t run_m2d_stream(Handle* h, const double* x, const float* sigl, const double* a, const float* qadd, float* q,
                           size_t smem) {
    static PerDevice attr;
    attr.get([&] {
        allow_max_dynamic_smem(m2d_stream_kernel<KT, NW>);
        return 1;
    });
    // the occupancy depends on this handle's tile size (smem)
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, m2d_stream_kernel<KT, NW>, NW * 32, smem);
    if (per_sm < 1) per_sm = 1;
    const long long ntiles = (h->NENK + NW * 8 - 1) / (NW * 8);
    long long grid = std::min<long long>(ntiles, (long long)h->sm_count * per_sm);
    m2d_stream_kernel<KT, NW><<<(int)grid, NW * 32, smem, h->stream>>>(h->d_active, x, sigl, a, qadd, h->d_mat, h->d_Ym2d, q,
                                                                        h->NENK, h->NI, h->NIpad, h->nm, h->nmpad, ntiles);
    return cudaGetLastError();
}

template <int MT, int NW>
cudaError_t run_d2m_stream(Handle* h, const float* psi, const double* xin, double alpha, double beta, double* out,
                           size_t smem) {
    static PerDevice attr;
    attr.get([&] {
        allow_max_dynamic_smem(d2m_stream_kernel<MT, NW>);
        return 1;
    });
    // the occupancy depends on this handle's tile size (smem)
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, d2m_stream_kernel<MT, NW>, NW * 32, smem);
    if (per_sm < 1) per_sm = 1;
    const long long ntiles = (h->NENK + NW * 8 - 1) / (NW * 8);
    long long grid = std::min<long long>(ntiles, (long long)h->sm_count * per_sm);
    d2m_stream_kernel<MT, NW><<<(int)grid, NW * 32, smem, h->stream>>>(h->d_active, psi, h->d_Yd2m, xin, alpha, beta, out,
                                                                        h->NENK, h->NI, h->NIpad, h->nm, h->nmpad, ntiles);
    return cudaGetLastError();
}

// Warps per CTA of the streaming contractions: 32 (one CTA and one copy of the constant operand per
// SM) unless LB_MOMENTS_WARPS=8 asks for four 256-thread CTAs.
int moments_warps() {
    static int nw = -1;
    if (nw < 0) {
        const char* e = std::getenv("LB_MOMENTS_WARPS");
        nw = (e && std::atoi(e) == 8) ? 8 : 32;
    }
    return nw;
}

constexpr size_t kStreamSmemLimit = 200 * 1024;

}  // namespace

int launch_m2d(Handle* h, const double* x, const float* sigl, const double* a, const float* qadd, float* q) {
    if (!sigl) sigl = h->d_sigl;
    if (moments_tc_enabled()) {
        Timer tt;
        timer_begin(h, LB_T_M2D, tt);
        const int rc = launch_m2d_tc(h, x, sigl, a, qadd, q);
        timer_end(h, tt);
        if (rc != LB_ERR_ARG) return rc;
    }
    const long long ntiles = (h->NENK + kTileN - 1) / kTileN;
    const int KT = h->nmpad / 16;
    const size_t smem_stream = (size_t)3 * h->NIpad * (h->nmpad + 8) * 2;
    Timer t;
    timer_begin(h, LB_T_M2D, t);
    cudaError_t e = cudaSuccess;
    if (KT <= 8 && smem_stream <= kStreamSmemLimit) {
        const bool w32 = moments_warps() == 32;
#define LB_M2D(K) e = w32 ? run_m2d_stream<K, 32>(h, x, sigl, a, qadd, q, smem_stream) \
                          : run_m2d_stream<K, 8>(h, x, sigl, a, qadd, q, smem_stream)
        switch (KT) {
            case 1: LB_M2D(1); break;
            case 2: LB_M2D(2); break;
            case 3: LB_M2D(3); break;
            case 4: LB_M2D(4); break;
            case 5: LB_M2D(5); break;
            case 6: LB_M2D(6); break;
            case 7: LB_M2D(7); break;
            default: LB_M2D(8); break;
        }
#undef LB_M2D
    } else {
        static PerDevice attr;
        attr.get([&] {
            allow_max_dynamic_smem(m2d_kernel);
            return 1;
        });
        const size_t smem = (size_t)3 * kTileN * smem_stride_words(h->nmpad) * 4;
        if (smem > 227 * 1024) { timer_end(h, t); return fail(h, LB_ERR_ARG, "m2d: too many moments for the shared-memory tile"); }
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, m2d_kernel, kThreads, smem);
        if (per_sm < 1) per_sm = 1;
        long long grid = std::min<long long>(ntiles, (long long)h->sm_count * per_sm);
        m2d_kernel<<<(int)grid, kThreads, smem, h->stream>>>(h->d_active, x, sigl, a, qadd, h->d_mat, h->d_Ym2d, q, h->NENK, h->NI,
                                                             h->NIpad, h->nm, h->nmpad, ntiles);
        e = cudaGetLastError();
    }
    timer_end(h, t);
    if (e != cudaSuccess) return cuda_fail(h, e, "m2d kernel launch");
    return LB_OK;
}

int launch_d2m(Handle* h, const float* psi, const double* xin, double alpha, double beta, double* out) {
    if (moments_tc_enabled()) {
        Timer tt;
        timer_begin(h, LB_T_D2M, tt);
        const int rc = launch_d2m_tc(h, psi, xin, alpha, beta, out);
        timer_end(h, tt);
        if (rc != LB_ERR_ARG) return rc;
    }
    const long long ntiles = (h->NENK + kTileN - 1) / kTileN;
    const int mtiles = h->nmpad / 16;
    const size_t smem_stream = (size_t)3 * h->nmpad * (h->NIpad + 8) * 2;
    Timer t;
    timer_begin(h, LB_T_D2M, t);
    cudaError_t e = cudaSuccess;
    int rc = LB_OK;
    if (smem_stream <= kStreamSmemLimit) {
        const bool w32 = moments_warps() == 32;
#define LB_D2M(M) e = w32 ? run_d2m_stream<M, 32>(h, psi, xin, alpha, beta, out, smem_stream) \
                          : run_d2m_stream<M, 8>(h, psi, xin, alpha, beta, out, smem_stream)
        if (mtiles <= 1) LB_D2M(1);
        else if (mtiles <= 3) LB_D2M(3);
        else if (mtiles <= 7) LB_D2M(7);
        else LB_D2M(16);
#undef LB_D2M
    } else {
        const size_t smem = (size_t)3 * kTileN * smem_stride_words(h->NIpad) * 4;
        if (smem > 227 * 1024) { timer_end(h, t); return fail(h, LB_ERR_ARG, "d2m: too many directions for the shared-memory tile"); }
        int per_sm = smem > 110 * 1024 ? 1 : 2;
        long long grid = std::min<long long>(ntiles, (long long)h->sm_count * per_sm);
        if (mtiles <= 1) rc = run_d2m<1>(h, psi, xin, alpha, beta, out, ntiles, (int)grid, smem);
        else if (mtiles <= 3) rc = run_d2m<3>(h, psi, xin, alpha, beta, out, ntiles, (int)grid, smem);
        else if (mtiles <= 7) rc = run_d2m<7>(h, psi, xin, alpha, beta, out, ntiles, (int)grid, smem);
        else rc = run_d2m<16>(h, psi, xin, alpha, beta, out, ntiles, (int)grid, smem);
        e = cudaGetLastError();
    }
    timer_end(h, t);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_fail(h, e, "d2m kernel launch");
    return LB_OK;
}

}  // namespace lb
