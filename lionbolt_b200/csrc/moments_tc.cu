// Moment contractions on the 5th-generation tensor cores (tcgen05, TMEM accumulators), sm_100a.
//
// Same products as moments.cu (D2M phi = (wY)^T psi, M2D q = Y Sigma phi; ScatteringAlgebra.f90:13-55
// factorised by the addition theorem), same split arithmetic: every FP32 operand value is split into
// three BF16 planes (hi + mid + lo) and the six products above 2^-24 of the leading term are
// accumulated in FP32.  Orientation: the MMA's M dimension is 128 DG nodes (one TMEM lane per node),
// so the epilogue reads one node per thread and every warp store writes 32 consecutive nodes of one
// direction (or moment) row: fully coalesced.
//
//   M2D: D[128 nodes][NH dirs] += A[128 nodes][K = moments] . B[NH dirs][K]^T   (N = NH <= 256)
//   D2M: D[128 nodes][48 moments] += A[128 nodes][K = dirs] . B[48 moments][K]^T (K streamed in chunks)
//
// Shared-memory operands use the K-major canonical layout without swizzle: for each 8-element K chunk
// the rows are contiguous 16-byte lines (8 rows = one 128-byte core matrix, SBO = 128 B) and
// consecutive K chunks are LBO bytes apart.  A (data) is produced by the CTA's threads (FP64 / FP32
// loads, scale, BF16 split, st.shared) and handed to the tensor core with fence.proxy.async; B (the
// constant Y planes) is staged once per CTA.  One thread issues the MMAs and commits them to an
// mbarrier; every wait is bounded and sets an error flag instead of hanging.
#include "lb_internal.h"
#include <algorithm>
#include <cstdlib>

namespace lb {

namespace {

constexpr int kTM = 128;                 // nodes per tile (MMA M)
constexpr long long kSpinLimit = 1LL << 22;   // polls before a wait is declared stuck (seconds at most)

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// tcgen05 shared-memory matrix descriptor: K-major, no swizzle (layout type 0), version 1.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: BF16 A and B (K-major), FP32 accumulator, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16_ss(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void bar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool bar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the MMA commit of the given phase.  Returns false (and raises *err) on timeout.
__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t parity, int* err) {
    for (long long it = 0; it < kSpinLimit; ++it) {
        if (bar_try_wait(bar, parity)) return true;
        if ((it & 1023) == 1023 && *(volatile int*)err) return false;
    }
    atomicExch(err, LB_ERR_TIMEOUT);
    return false;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = __uint_as_float(r[k]);
}

// The warp calling this allocates ncols TMEM columns (power of two >= 32) and publishes the base.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_free(uint32_t base, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols) : "memory");
}

// (v0..v7) -> three 16-byte BF16 lines (hi, mid, lo)
__device__ __forceinline__ void split8(const float (&v)[8], uint4& hi, uint4& mid, uint4& lo) {
    uint32_t h[4], m[4], l[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const __nv_bfloat162 a = __floats2bfloat162_rn(v[2 * k], v[2 * k + 1]);
        const float2 fa = __bfloat1622float2(a);
        const float r0 = v[2 * k] - fa.x, r1 = v[2 * k + 1] - fa.y;
        const __nv_bfloat162 b = __floats2bfloat162_rn(r0, r1);
        const float2 fb = __bfloat1622float2(b);
        const __nv_bfloat162 c = __floats2bfloat162_rn(r0 - fb.x, r1 - fb.y);
        h[k] = *reinterpret_cast<const uint32_t*>(&a);
        m[k] = *reinterpret_cast<const uint32_t*>(&b);
        l[k] = *reinterpret_cast<const uint32_t*>(&c);
    }
    hi = make_uint4(h[0], h[1], h[2], h[3]);
    mid = make_uint4(m[0], m[1], m[2], m[3]);
    lo = make_uint4(l[0], l[1], l[2], l[3]);
}

// plane pairs (A plane, B plane) of the six split products, small terms first
__constant__ int kProdA[6] = {2, 1, 0, 1, 0, 0};
__constant__ int kProdB[6] = {0, 1, 2, 0, 1, 0};

// Copies rows [r0, r0 + nrows) of a [3][rows][cols] BF16 plane set (row-major, cols % 8 == 0) into
// the K-major canonical layout: plane p, K chunk c, row r at  p*pstride + c*(nrows*16) + r*16 bytes.
// Rows past `rows` are zero.
__device__ void stage_kmajor(const __nv_bfloat16* __restrict__ g, int rows, int cols, int r0, int nrows,
                             unsigned char* s, size_t pstride) {
    const int cc = cols / 8;
    const int total = 3 * nrows * cc;
    for (int u = threadIdx.x; u < total; u += blockDim.x) {
        const int p = u / (nrows * cc);
        const int rem = u % (nrows * cc);
        const int r = rem / cc, c = rem % cc;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if (r0 + r < rows) v = __ldg(reinterpret_cast<const uint4*>(g + ((size_t)p * rows + r0 + r) * cols) + c);
        *reinterpret_cast<uint4*>(s + p * pstride + (size_t)c * nrows * 16 + (size_t)r * 16) = v;
    }
}

// ---------------------------------------------------------------------------------------------
// M2D: q[i][n] = sum_j Y[i][j] xt[j][n] (+ qadd[i][n]),  xt[j][n] = sigl[mat(n)][j] x[j][n] + a[j][n].
// CTA = 128 threads (thread t owns node tile*128 + t), directions [half*NH, half*NH + NH).
// ---------------------------------------------------------------------------------------------
template <int KT>
__global__ void __launch_bounds__(128, 2) m2d_tc_kernel(const int* __restrict__ active, const double* __restrict__ x,
                                                      const float* __restrict__ sigl, const double* __restrict__ add,
                                                      const float* __restrict__ qadd, const int* __restrict__ mat,
                                                      const __nv_bfloat16* __restrict__ Y, float* __restrict__ q,
                                                      long long NENK, int NI, int NIpad, int nm, int nmpad, int NH,
                                                      int nhalves, uint32_t tmem_cols, long long ntiles, int* err) {
    if (active && *active == 0) return;
    extern __shared__ __align__(1024) unsigned char sm[];
    const int tid = threadIdx.x, warp = tid >> 5;
    const size_t bplane = (size_t)NH * nmpad * 2;     // bytes per B plane
    const size_t aplane = (size_t)kTM * nmpad * 2;    // bytes per A plane
    unsigned char* sB = sm;
    unsigned char* sA = sm + ((3 * bplane + 1023) / 1024) * 1024;
    uint64_t* bar = reinterpret_cast<uint64_t*>(sA + 3 * aplane);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
    const int half = blockIdx.x % nhalves;
    stage_kmajor(Y, NIpad, nmpad, half * NH, NH, sB, bplane);
    if (tid == 0) bar_init(bar, 1);
    if (warp == 0) tmem_alloc(tslot, tmem_cols);
    fence_async_smem();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tmem = *tslot;
    const uint32_t idesc = idesc_bf16(kTM, NH);
    const uint32_t lboA = kTM * 16, lboB = (uint32_t)NH * 16;
    const uint32_t aBase = smem_u32(sA), bBase = smem_u32(sB);
    constexpr int NMP = KT * 16;
    uint32_t phase = 0;
    bool ok = true;
    const long long tstep = gridDim.x / nhalves;
    // raw inputs of the current tile, loaded one tile ahead: x (or the additive source) per moment
    double cur[NMP];
    auto fetch = [&](long long tl, double (&r)[NMP]) {
        const long long nn = tl * kTM + tid;
        const double* src = x ? x : add;
#pragma unroll
        for (int j = 0; j < NMP; ++j) r[j] = (tl < ntiles && nn < NENK && j < nm) ? __ldcs(&src[(size_t)j * NENK + nn]) : 0.0;
    };
    fetch(blockIdx.x / nhalves, cur);
    for (long long tile = blockIdx.x / nhalves; tile < ntiles && ok; tile += tstep) {
        const long long n = tile * kTM + tid;
        const bool valid = n < NENK;
        const int m = valid ? __ldg(&mat[n >> 2]) : 0;
        // A: xt rows of this tile, split into BF16 planes
#pragma unroll
        for (int c = 0; c < NMP / 8; ++c) {
            float v[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int j = c * 8 + k;
                double s = 0.0;
                if (valid && j < nm) {
                    if (x) {
                        s = (double)__ldg(&sigl[(size_t)m * nmpad + j]) * cur[j];
                        if (add) s += __ldcs(&add[(size_t)j * NENK + n]);
                    } else {
                        s = cur[j];
                    }
                }
                v[k] = (float)s;
            }
            uint4 hi, mid, lo;
            split8(v, hi, mid, lo);
            unsigned char* row = sA + (size_t)c * kTM * 16 + (size_t)tid * 16;
            *reinterpret_cast<uint4*>(row) = hi;
            *reinterpret_cast<uint4*>(row + aplane) = mid;
            *reinterpret_cast<uint4*>(row + 2 * aplane) = lo;
        }
        // next tile's inputs are requested now and arrive during this tile's MMAs and epilogue
        fetch(tile + tstep, cur);
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc_after_sync();
            for (int ks = 0; ks < KT; ++ks)
                for (int pr = 0; pr < 6; ++pr) {
                    const uint64_t da = sdesc(aBase + kProdA[pr] * (uint32_t)aplane + ks * 2 * lboA, lboA, 128);
                    const uint64_t db = sdesc(bBase + kProdB[pr] * (uint32_t)bplane + ks * 2 * lboB, lboB, 128);
                    mma_bf16_ss(tmem, da, db, idesc, (ks | pr) ? 1u : 0u);
                }
            mma_commit(bar);
        }
        ok = __syncthreads_and(bar_wait(bar, phase, err));
        phase ^= 1u;
        tc_after_sync();
        if (ok) {
            // epilogue: warp w reads TMEM lanes 32w..32w+31 = its threads' nodes
            const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
            for (int c0 = 0; c0 < NH; c0 += 16) {
                float v[16];
                tmem_ld16(lane_base + (uint32_t)c0, v);
                if (valid) {
#pragma unroll
                    for (int k = 0; k < 16; ++k) {
                        const int i = half * NH + c0 + k;
                        if (i < NI) {
                            float o = v[k];
                            if (qadd) o += qadd[(size_t)i * NENK + n];
                            __stcs(&q[(size_t)i * NENK + n], o);
                        }
                    }
                }
            }
        }
        tc_before_sync();
        ok = __syncthreads_and(ok && !*(volatile int*)err);
        tc_after_sync();
    }
    tc_before_sync();
    __syncthreads();
    if (warp == 0) tmem_free(tmem, tmem_cols);
}

// ---------------------------------------------------------------------------------------------
// D2M: z[j][n] = sum_i Dw[j][i] psi[i][n];  out = alpha * xin + beta * z.
// CTA = 256 threads; psi is streamed in K chunks of 48 directions (double-buffered A planes):
// threads t and t + 128 share node tile*128 + (t & 127) and split the chunk's directions, and in the
// epilogue the moments, in halves.  KT = nmpad / 16.
// ---------------------------------------------------------------------------------------------
constexpr int kKC = 48;   // directions per K chunk (3 MMA K-steps)

template <int KT>
__global__ void __launch_bounds__(256, 1) d2m_tc_kernel(const int* __restrict__ active, const float* __restrict__ psi,
                                                      const __nv_bfloat16* __restrict__ Dw, const double* xin,
                                                      double alpha, double beta, double* out, long long NENK, int NI,
                                                      int NIpad, int nm, int nmpad, long long ntiles, int* err) {
    if (active && *active == 0) return;
    extern __shared__ __align__(1024) unsigned char sm[];
    const int tid = threadIdx.x, warp = tid >> 5;
    const int row = tid & 127, side = tid >> 7;
    const int NKpad = (NIpad + kKC - 1) / kKC * kKC;         // directions padded to whole chunks
    const size_t bplane = (size_t)nmpad * NKpad * 2;         // B: [3][K chunks][nmpad rows][16 B]
    const size_t aplane = (size_t)kTM * kKC * 2;             // A chunk: [3][6 K chunks][128 rows][16 B]
    unsigned char* sB = sm;
    unsigned char* sA0 = sm + ((3 * bplane + 1023) / 1024) * 1024;
    unsigned char* sA1 = sA0 + ((3 * aplane + 1023) / 1024) * 1024;
    uint64_t* bar = reinterpret_cast<uint64_t*>(sA1 + 3 * aplane);   // [2]
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 2);
    // B = Dw planes [3][nmpad][NIpad] (row-major) staged K-major: rows = moments, K = directions
    {
        const int cc = NKpad / 8;
        const int total = 3 * nmpad * cc;
        for (int u = tid; u < total; u += blockDim.x) {
            const int p = u / (nmpad * cc);
            const int rem = u % (nmpad * cc);
            const int r = rem / cc, c = rem % cc;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (c * 8 < NIpad) v = __ldg(reinterpret_cast<const uint4*>(Dw + ((size_t)p * nmpad + r) * NIpad) + c);
            *reinterpret_cast<uint4*>(sB + p * bplane + (size_t)c * nmpad * 16 + (size_t)r * 16) = v;
        }
    }
    if (tid == 0) {
        bar_init(&bar[0], 1);
        bar_init(&bar[1], 1);
    }
    if (warp == 0) tmem_alloc(tslot, 64);
    fence_async_smem();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tmem = *tslot;
    const uint32_t idesc = idesc_bf16(kTM, nmpad);
    const uint32_t lboA = kTM * 16, lboB = (uint32_t)nmpad * 16;
    const uint32_t bBase = smem_u32(sB);
    const int nchunks = NKpad / kKC;
    uint32_t uses[2] = {0u, 0u};   // completed commits per buffer
    bool ok = true;
    // this thread's 24 psi values of a chunk (3 K lines of 8 directions), loaded one chunk ahead
    float cur[24];
    auto fetch = [&](long long tl, int chk, float (&r)[24]) {
        const long long nn = tl * kTM + row;
        const bool vv = tl < ntiles && nn < NENK;
#pragma unroll
        for (int u = 0; u < 24; ++u) {
            const int i = chk * kKC + side * 24 + u;
            r[u] = (vv && i < NI) ? __ldcs(&psi[(size_t)i * NENK + nn]) : 0.f;
        }
    };
    fetch(blockIdx.x, 0, cur);
    for (long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const long long n = tile * kTM + row;
        const bool valid = n < NENK;
        for (int ch = 0; ch < nchunks && ok; ++ch) {
            const int b = ch & 1;
            unsigned char* sA = b ? sA1 : sA0;
            float nxt[24];
            if (ch + 1 < nchunks) fetch(tile, ch + 1, nxt);
            else fetch(tile + gridDim.x, 0, nxt);
            // the buffer's previous MMAs must be done before it is overwritten
            if (uses[b] > 0) {
                ok = __syncthreads_and(bar_wait(&bar[b], (uses[b] - 1) & 1u, err));
                if (!ok) break;
            }
#pragma unroll
            for (int cl = 0; cl < 3; ++cl) {
                const int c = side * 3 + cl;
                float v[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) v[k] = cur[cl * 8 + k];
                uint4 hi, mid, lo;
                split8(v, hi, mid, lo);
                unsigned char* r = sA + (size_t)c * kTM * 16 + (size_t)row * 16;
                *reinterpret_cast<uint4*>(r) = hi;
                *reinterpret_cast<uint4*>(r + aplane) = mid;
                *reinterpret_cast<uint4*>(r + 2 * aplane) = lo;
            }
#pragma unroll
            for (int u = 0; u < 24; ++u) cur[u] = nxt[u];
            fence_async_smem();
            __syncthreads();
            if (tid == 0) {
                tc_after_sync();
                const uint32_t aBase = smem_u32(sA);
                for (int ks = 0; ks < kKC / 16; ++ks)
                    for (int pr = 0; pr < 6; ++pr) {
                        const uint64_t da = sdesc(aBase + kProdA[pr] * (uint32_t)aplane + ks * 2 * lboA, lboA, 128);
                        const uint64_t db = sdesc(bBase + kProdB[pr] * (uint32_t)bplane +
                                                      (uint32_t)(ch * (kKC / 8) + ks * 2) * lboB, lboB, 128);
                        mma_bf16_ss(tmem, da, db, idesc, (ch | ks | pr) ? 1u : 0u);
                    }
                mma_commit(&bar[b]);
            }
            ++uses[b];
        }
        if (!ok) break;
        // epilogue operands: this thread's half of the moments (side * KT*8 ..), requested before
        // the wait so that their latency overlaps the last MMAs
        constexpr int CPS = KT * 8;   // columns per side
        double xv[CPS];
#pragma unroll
        for (int u = 0; u < CPS; ++u) {
            const int j = side * CPS + u;
            xv[u] = (xin && valid && j < nm) ? xin[(size_t)j * NENK + n] : 0.0;
        }
        // all chunks of the tile: wait for the last commit of each buffer
        for (int b = 0; b < 2 && ok; ++b)
            if (uses[b] > 0) ok = __syncthreads_and(bar_wait(&bar[b], (uses[b] - 1) & 1u, err));
        tc_after_sync();
        if (ok) {
            // warps w and w + 4 share TMEM lanes 32(w%4)..; each reads its side's columns
            const uint32_t lane_base = tmem + ((uint32_t)((warp & 3) * 32) << 16);
#pragma unroll
            for (int g = 0; g < KT; ++g) {
                float v[8];
                tmem_ld8(lane_base + (uint32_t)(side * CPS + g * 8), v);
                if (valid) {
#pragma unroll
                    for (int k = 0; k < 8; ++k) {
                        const int j = side * CPS + g * 8 + k;
                        if (j < nm) out[(size_t)j * NENK + n] = beta * (double)v[k] + alpha * xv[g * 8 + k];
                    }
                }
            }
        }
        tc_before_sync();
        ok = __syncthreads_and(ok && !*(volatile int*)err);
        tc_after_sync();
    }
    tc_before_sync();
    __syncthreads();
    if (warp == 0) tmem_free(tmem, 64);
}

size_t m2d_tc_smem(int NH, int nmpad) {
    const size_t b = ((3 * (size_t)NH * nmpad * 2 + 1023) / 1024) * 1024;
    return b + 3 * (size_t)kTM * nmpad * 2 + 64;
}

size_t d2m_tc_smem(int NIpad, int nmpad) {
    const int NKpad = (NIpad + kKC - 1) / kKC * kKC;
    const size_t b = ((3 * (size_t)nmpad * NKpad * 2 + 1023) / 1024) * 1024;
    const size_t a = ((3 * (size_t)kTM * kKC * 2 + 1023) / 1024) * 1024;
    return b + a + 3 * (size_t)kTM * kKC * 2 + 64;
}

int* tc_error_flag() {
    static int* flag = nullptr;
    if (!flag && cudaMalloc(&flag, sizeof(int)) == cudaSuccess) cudaMemset(flag, 0, sizeof(int));
    return flag;
}

}  // namespace

bool moments_tc_enabled() {
    static int on = -1;
    if (on < 0) {
        const char* e = std::getenv("LB_MOMENTS_TC");
        on = (e && *e == '0') ? 0 : 1;
    }
    return on == 1;
}

// Returns LB_ERR_ARG when the shape does not fit the tensor-core kernels (caller falls back).
int launch_m2d_tc(Handle* h, const double* x, const float* sigl, const double* a, const float* qadd, float* q) {
    const int nhalves = h->NIpad > 256 ? 2 : 1;
    const int NH = ((h->NIpad + nhalves - 1) / nhalves + 15) / 16 * 16;
    if (NH > 256 || h->nmpad % 16 || h->nmpad > 64 || h->NIpad % 8) return LB_ERR_ARG;
    const uint32_t cols = NH <= 32 ? 32 : NH <= 64 ? 64 : NH <= 128 ? 128 : 256;
    // at most two CTAs per SM: their TMEM (<= 2 x 256 columns) always fits, so no allocation waits
    const size_t smem = std::max<size_t>(m2d_tc_smem(NH, h->nmpad), 80 * 1024);
    if (smem > 113 * 1024) return LB_ERR_ARG;
    int* err = tc_error_flag();
    if (!err) return LB_ERR_OOM;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(m2d_tc_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 113 * 1024);
        cudaFuncSetAttribute(m2d_tc_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 113 * 1024);
        cudaFuncSetAttribute(m2d_tc_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, 113 * 1024);
        cudaFuncSetAttribute(m2d_tc_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, 113 * 1024);
        attr = true;
    }
    const long long ntiles = (h->NENK + kTM - 1) / kTM;
    long long grid = std::min<long long>(ntiles * nhalves, (long long)h->sm_count * 2);
    grid = std::max<long long>(nhalves, grid / nhalves * nhalves);
    const int KT = h->nmpad / 16;
#define LB_M2DTC(K)                                                                                               \
    m2d_tc_kernel<K><<<(int)grid, 128, smem, h->stream>>>(h->d_active, x, sigl, a, qadd, h->d_mat, h->d_Ym2d, q, h->NENK, \
                                                           h->NI, h->NIpad, h->nm, h->nmpad, NH, nhalves, cols, ntiles, err)
    switch (KT) {
        case 1: LB_M2DTC(1); break;
        case 2: LB_M2DTC(2); break;
        case 3: LB_M2DTC(3); break;
        default: LB_M2DTC(4); break;
    }
#undef LB_M2DTC
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LB_OK : cuda_fail(h, e, "m2d tensor-core kernel");
}

int launch_d2m_tc(Handle* h, const float* psi, const double* xin, double alpha, double beta, double* out) {
    if (h->nmpad > 64 || h->nmpad % 16 || h->NIpad % 8) return LB_ERR_ARG;
    // at most two CTAs per SM (2 x 64 TMEM columns)
    const size_t smem = std::max<size_t>(d2m_tc_smem(h->NIpad, h->nmpad), 80 * 1024);
    if (smem > 227 * 1024) return LB_ERR_ARG;
    int* err = tc_error_flag();
    if (!err) return LB_ERR_OOM;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(d2m_tc_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        cudaFuncSetAttribute(d2m_tc_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        cudaFuncSetAttribute(d2m_tc_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        cudaFuncSetAttribute(d2m_tc_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        attr = true;
    }
    const long long ntiles = (h->NENK + kTM - 1) / kTM;
    const long long grid = std::min<long long>(ntiles, (long long)h->sm_count);
#define LB_D2MTC(K)                                                                                        \
    d2m_tc_kernel<K><<<(int)grid, 256, smem, h->stream>>>(h->d_active, psi, h->d_Yd2m, xin, alpha, beta, out, \
                                                           h->NENK, h->NI, h->NIpad, h->nm, h->nmpad, ntiles, err)
    switch (h->nmpad / 16) {
        case 1: LB_D2MTC(1); break;
        case 2: LB_D2MTC(2); break;
        case 3: LB_D2MTC(3); break;
        default: LB_D2MTC(4); break;
    }
#undef LB_D2MTC
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LB_OK : cuda_fail(h, e, "d2m tensor-core kernel");
}

// Reads and clears the tensor-core kernels' timeout flag (synchronises the handle's stream).
int moments_tc_status(Handle* h) {
    int* err = tc_error_flag();
    if (!err) return LB_OK;
    int v = 0;
    cudaStreamSynchronize(h->stream);
    cudaMemcpy(&v, err, sizeof(int), cudaMemcpyDeviceToHost);
    if (v) {
        cudaMemset(err, 0, sizeof(int));
        return fail(h, LB_ERR_TIMEOUT, "tensor-core moment kernel: MMA completion wait timed out");
    }
    return LB_OK;
}

}  // namespace lb
