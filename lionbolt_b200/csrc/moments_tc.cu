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
// constant Y planes) is staged once per CTA.  Each kernel is warp-specialised (producer warps, an MMA
// warp whose lane 0 issues every tcgen05.mma, epilogue warps) with double-buffered operands and
// accumulators synchronised by mbarriers; every wait is bounded and sets an error flag instead of
// hanging.
#include "lb_internal.h"
#include <cuda.h>
#include <algorithm>
#include <cstdlib>
#include <cstring>

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
__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t parity, int* err, long long limit = kSpinLimit) {
    for (long long it = 0; it < limit; ++it) {
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

__device__ __forceinline__ void bar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Tensor-memory-accelerator load of a 2-D box (no multicast): the mbarrier completes when its bytes land.
__device__ __forceinline__ void bar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// Tensor-memory-accelerator store of a 2-D box from shared memory (a bulk group; parts of the box outside
// the tensor are not written).
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, const void* src, int x, int y) {
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%2, %3}], [%1];"
                 ::"l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(src)), "r"(x), "r"(y)
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// ---------------------------------------------------------------------------------------------
// M2D: q[i][n] = sum_j Y[i][j] xt[j][n] (+ qadd[i][n]),  xt[j][n] = sigl[mat(n)][j] x[j][n] + a[j][n].
// One CTA per SM, warp-specialised, directions [half*NH, half*NH + NH) of every tile it takes:
//   warps 0-7   producers: threads t and t + 128 read node tile*128 + (t & 127), half of its moments
//               each, split them into BF16 planes and write the A buffer (two buffers);
//   warps 8-19  epilogue: warps 8+e, 12+e and 16+e read TMEM lanes 32e.. (the tile's nodes), a third
//               of the direction columns each, and write q rows (two accumulators);
//   warp 20     lane 0 issues the MMAs; the warp owns the TMEM allocation.
// Barriers per buffer b: full[b] (producers -> MMA), done[b] (MMA commit -> producers, epilogue),
// empty[b] (epilogue -> MMA).  The k-th use of a buffer waits on phase parity k & 1.
// ---------------------------------------------------------------------------------------------
constexpr int kM2dEpi = 12;                          // epilogue warps (three per TMEM lane quarter)
constexpr int kM2dMma = 8 + kM2dEpi;                 // the MMA warp
constexpr int kM2dThreads = 32 * (kM2dMma + 1);
constexpr int kM2dTma = kM2dMma + 1;                 // MODE 2: the warp whose lane 0 loads the moment tiles
constexpr int kM2dThreadsTma = 32 * (kM2dTma + 1);

// MODE 0: per-thread output stores; 1: TMA output stores (two staging buffers per epilogue warp); 2: TMA
// output stores (one buffer per warp) and the moment tiles x[0..nm)[128 nodes] brought into a two-stage
// shared-memory ring by TMA, from which the producers read (nodes past NENK arrive as zeros).
template <int KT, int MODE>
__global__ void __launch_bounds__(MODE == 2 ? kM2dThreadsTma : kM2dThreads, 1) m2d_tc_kernel(
                                                      const __grid_constant__ CUtensorMap q_map,
                                                      const __grid_constant__ CUtensorMap x_map,
                                                      const int* __restrict__ active, const double* __restrict__ x,
                                                      const float* __restrict__ sigl, const double* __restrict__ add,
                                                      const float* __restrict__ qadd, const int* __restrict__ mat,
                                                      const __nv_bfloat16* __restrict__ Y, float* __restrict__ q,
                                                      long long NENK, int NI, int NIpad, int nm, int nmpad, int NH,
                                                      int nhalves, long long ntiles, int* err) {
    if (active && *active == 0) return;
    extern __shared__ __align__(1024) unsigned char sm[];
    constexpr int NMP = KT * 16;
    const int tid = threadIdx.x, warp = tid >> 5;
    const size_t bplane = (size_t)NH * nmpad * 2;
    const size_t aplane = (size_t)kTM * nmpad * 2;
    const size_t abuf = ((3 * aplane + 1023) / 1024) * 1024;
    unsigned char* sB = sm;
    unsigned char* sA = sm + ((3 * bplane + 1023) / 1024) * 1024;   // [2] buffers of 3 planes
    uint64_t* full = reinterpret_cast<uint64_t*>(sA + 2 * abuf);
    uint64_t* done = full + 2;
    uint64_t* empty = full + 4;
    uint64_t* xfull = full + 6;     // MODE 2: [2] moment stages loaded
    uint64_t* xempty = full + 8;    // MODE 2: [2] moment stages read
    uint32_t* tslot = reinterpret_cast<uint32_t*>(full + 10);
    // MODE >= 1: per epilogue warp NB 2 KB staging buffers [16 directions][32 nodes] for the TMA stores
    constexpr int NB = MODE == 2 ? 1 : 2;
    float* sS = reinterpret_cast<float*>(sA + 2 * abuf + 1024);
    const size_t xbuf = (size_t)kTM * nm * 8;                                    // MODE 2: one moment stage
    unsigned char* sX = sA + 2 * abuf + 1024 + (size_t)kM2dEpi * NB * 2048;       // MODE 2: [2] stages
    const int half = blockIdx.x % nhalves;
    stage_kmajor(Y, NIpad, nmpad, half * NH, NH, sB, bplane);
    if (tid == 0) {
        for (int k = 0; k < 2; ++k) {
            bar_init(&full[k], 256);
            bar_init(&done[k], 1);
            bar_init(&empty[k], 32 * kM2dEpi);
        }
        if (MODE == 2)
            for (int k = 0; k < 2; ++k) {
                bar_init(&xfull[k], 1);
                bar_init(&xempty[k], 256);
            }
    }
    if (warp == kM2dMma) tmem_alloc(tslot, 512);
    fence_async_smem();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tmem = *tslot;
    const long long t0 = blockIdx.x / nhalves, tstep = gridDim.x / nhalves;
    if (warp < 8) {
        // ---- producers: threads t and t + 128 share node tile*128 + (t & 127), each half the moments ----
        constexpr int HM = NMP / 2;
        const int r = tid & 127, side = tid >> 7;
        const double* src = x ? x : add;
        // the node's material (it selects the sigma row) is loaded one tile ahead, off the tile's load chain
        int m_next = (t0 * kTM + r < NENK) ? __ldg(&mat[(t0 * kTM + r) >> 2]) : 0;
        int it = 0;
        for (long long tile = t0; tile < ntiles; tile += tstep, ++it) {
            const int b = it & 1;
            const uint32_t u = (uint32_t)(it >> 1);
            const long long n = tile * kTM + r;
            const bool valid = n < NENK;
            const int m = valid ? m_next : 0;
            {
                const long long nn = (tile + tstep) * kTM + r;
                m_next = nn < NENK ? __ldg(&mat[nn >> 2]) : 0;
            }
            double raw[HM];
            if (MODE == 2) {
                // the tile's moments from the stage, then the stage back to the TMA: the proxy fence orders
                // these generic reads before its next (async-proxy) write into the stage
                const int xs = it & 1;
                if (!bar_wait(&xfull[xs], (uint32_t)(it >> 1) & 1u, err)) break;
                const double* X = reinterpret_cast<const double*>(sX + xs * xbuf) + (size_t)(side * HM) * kTM + r;
                const int jn = nm - side * HM;
#pragma unroll
                for (int k = 0; k < HM; ++k) raw[k] = k < jn ? X[(size_t)k * kTM] : 0.0;
                fence_async_smem();
                bar_arrive(&xempty[xs]);
            } else {
                // one pointer stepped by a row (NENK) per moment instead of a 64-bit index per load
                const double* sp = src + (size_t)(side * HM) * (size_t)NENK + (valid ? n : 0);
                const int jn = valid ? nm - side * HM : 0;   // moments of this half that exist
#pragma unroll
                for (int k = 0; k < HM; ++k) {
                    raw[k] = k < jn ? __ldcs(sp) : 0.0;
                    sp += NENK;
                }
            }
            if (u > 0 && !bar_wait(&done[b], (u - 1) & 1u, err)) break;
            unsigned char* A = sA + b * abuf;
            // this half's sigma_l(j) row of the node's material (the table is padded to nmpad with zeros, and
            // raw[] is zero past the moments that exist, so no per-value bounds test is needed)
            const float* sg = sigl + (size_t)m * nmpad + side * HM;
            const int jn = valid ? nm - side * HM : 0;
            const double* ap = (x && add && valid) ? add + (size_t)(side * HM) * (size_t)NENK + n : nullptr;
#pragma unroll
            for (int cl = 0; cl < HM / 8; ++cl) {
                float v[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const int kk = cl * 8 + k;
                    double sv = raw[kk];
                    if (x) {
                        sv = (double)__ldg(&sg[kk]) * sv;
                        if (ap && kk < jn) sv += __ldcs(ap + (size_t)kk * (size_t)NENK);
                    }
                    v[k] = (float)sv;
                }
                uint4 hi, mid, lo;
                split8(v, hi, mid, lo);
                unsigned char* row = A + (size_t)(side * (HM / 8) + cl) * kTM * 16 + (size_t)r * 16;
                *reinterpret_cast<uint4*>(row) = hi;
                *reinterpret_cast<uint4*>(row + aplane) = mid;
                *reinterpret_cast<uint4*>(row + 2 * aplane) = lo;
            }
            fence_async_smem();
            bar_arrive(&full[b]);
        }
    } else if (warp < kM2dMma) {
        // ---- epilogue: warps w, w + 4 and w + 8 share TMEM lanes 32(w%4).. and split the columns ----
        const int e = warp - 8;
        const int r = (e & 3) * 32 + (tid & 31);
        const int ngr = NH / 16, per = (ngr + kM2dEpi / 4 - 1) / (kM2dEpi / 4);
        const int g0 = (e >> 2) * per, g1 = min(ngr, g0 + per);
        const uint32_t lane_base = tmem + ((uint32_t)((e & 3) * 32) << 16);
        const int lane = tid & 31;
        float* stage = sS + (size_t)e * NB * 512;    // MODE >= 1: this warp's NB [16][32] buffers
        int sidx = 0;
        int it = 0;
        for (long long tile = t0; tile < ntiles; tile += tstep, ++it) {
            const int b = it & 1;
            const uint32_t u = (uint32_t)(it >> 1);
            if (!bar_wait(&done[b], u & 1u, err)) break;
            tc_after_sync();
            const long long n = tile * kTM + r;
            const bool valid = n < NENK;
            for (int g = g0; g < g1; ++g) {
                float v[16];
                tmem_ld16(lane_base + (uint32_t)(b * 256 + g * 16), v);
                if (MODE >= 1) {
                    // the warp's 32 nodes x 16 directions through shared memory and one TMA store (nodes past
                    // NENK and directions past NI lie outside the tensor and are not written)
                    float* st = stage + sidx * 512;
                    if (lane == 0) {
                        if (NB == 2) asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
                        else asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
                    }
                    __syncwarp();
#pragma unroll
                    for (int k = 0; k < 16; ++k) st[k * 32 + lane] = v[k];
                    fence_async_smem();
                    __syncwarp();
                    if (lane == 0) tma_store_2d(&q_map, st, (int)(tile * kTM) + (e & 3) * 32, half * NH + g * 16);
                    sidx = (sidx + 1) % NB;
                    continue;
                }
                if (valid) {
                    const int i0 = half * NH + g * 16;
                    const size_t o0 = (size_t)i0 * (size_t)NENK + (size_t)n;
                    // plain (write-back) stores: the tile's 512-byte row pieces stay in L2 until the
                    // neighbouring tiles' pieces join them (evict-first stores: 5 % slower)
                    if (!qadd && i0 + 16 <= NI) {
                        // the common case, one pointer stepped by a row per direction
                        float* qp = q + o0;
#pragma unroll
                        for (int k = 0; k < 16; ++k) {
                            *qp = v[k];
                            qp += NENK;
                        }
                    } else {
#pragma unroll
                        for (int k = 0; k < 16; ++k) {
                            if (i0 + k < NI) {
                                const size_t o = o0 + (size_t)k * (size_t)NENK;
                                q[o] = qadd ? v[k] + qadd[o] : v[k];
                            }
                        }
                    }
                }
            }
            tc_before_sync();
            bar_arrive(&empty[b]);
        }
        // the staging buffers stay in use until the stores have read them
        if (MODE >= 1 && lane == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    } else if (warp == kM2dMma && (tid & 31) == 0) {
        // ---- MMA issue ----
        const uint32_t idesc = idesc_bf16(kTM, NH);
        const uint32_t lboA = kTM * 16, lboB = (uint32_t)NH * 16;
        const uint32_t aBase = smem_u32(sA), bBase = smem_u32(sB);
        int it = 0;
        for (long long tile = t0; tile < ntiles; tile += tstep, ++it) {
            const int b = it & 1;
            const uint32_t u = (uint32_t)(it >> 1);
            if (!bar_wait(&full[b], u & 1u, err)) break;
            if (u > 0 && !bar_wait(&empty[b], (u - 1) & 1u, err)) break;
            tc_after_sync();
            const uint32_t a0 = aBase + b * (uint32_t)abuf;
            for (int ks = 0; ks < KT; ++ks)
                for (int pr = 0; pr < 6; ++pr) {
                    const uint64_t da = sdesc(a0 + kProdA[pr] * (uint32_t)aplane + ks * 2 * lboA, lboA, 128);
                    const uint64_t db = sdesc(bBase + kProdB[pr] * (uint32_t)bplane + ks * 2 * lboB, lboB, 128);
                    mma_bf16_ss(tmem + b * 256, da, db, idesc, (ks | pr) ? 1u : 0u);
                }
            mma_commit(&done[b]);
        }
    } else if (MODE == 2 && warp == kM2dTma && (tid & 31) == 0) {
        // ---- moment tiles by TMA, up to two ahead of the producers ----
        int it = 0;
        for (long long tile = t0; tile < ntiles; tile += tstep, ++it) {
            const int xs = it & 1;
            if (it >= 2 && !bar_wait(&xempty[xs], (uint32_t)((it >> 1) - 1) & 1u, err)) break;
            bar_expect_tx(&xfull[xs], (uint32_t)xbuf);
            tma_load_2d(sX + xs * xbuf, &x_map, (int)(tile * kTM), 0, &xfull[xs]);
        }
    }
    tc_before_sync();
    __syncthreads();
    if (warp == kM2dMma) tmem_free(tmem, 512);
}

// ---------------------------------------------------------------------------------------------
// D2M: z[j][n] = sum_i Dw[j][i] psi[i][n];  out = alpha * xin + beta * z.  KT = nmpad / 16.
// One CTA per SM, warp-specialised; psi streams in K chunks of 48 directions through a ring of
// kStages A buffers:
//   warps 0..8S-1  producers, S = kD2mSets sets of 8 warps taking alternate chunks (S chunks of loads
//               in flight): threads t and t + 128 of a set share node tile*128 + (t & 127), each loads
//               and splits 24 directions of the chunk;
//   next 4 warps  epilogue (TMEM lanes 32(w%4)..): out rows of the tile (two accumulators);
//   last warp   lane 0 issues the MMAs; the warp owns the TMEM allocation.
// The leading split product and the five smaller ones accumulate separately, as in d2m_tma_kernel.
// ---------------------------------------------------------------------------------------------
constexpr int kKC = 48;       // directions per K chunk (3 MMA K-steps)
constexpr int kStages = 3;    // A ring depth
constexpr int kD2mSets = 2;                     // producer sets of 8 warps, taking alternate chunks
constexpr int kD2mEpi = 8 * kD2mSets;           // first of the 4 epilogue warps
constexpr int kD2mMma = kD2mEpi + 4;            // the MMA warp
constexpr int kD2mThreads = 32 * (kD2mMma + 1);

template <int KT>
__global__ void __launch_bounds__(kD2mThreads, 1) d2m_tc_kernel(const int* __restrict__ active, const float* __restrict__ psi,
                                                      const __nv_bfloat16* __restrict__ Dw, const double* xin,
                                                      double alpha, double beta, double* out, long long NENK, int NI,
                                                      int NIpad, int nm, int nmpad, long long ntiles, int* err) {
    if (active && *active == 0) return;
    extern __shared__ __align__(1024) unsigned char sm[];
    const int tid = threadIdx.x, warp = tid >> 5;
    const int NKpad = (NIpad + kKC - 1) / kKC * kKC;
    const size_t bplane = (size_t)nmpad * NKpad * 2;
    const size_t aplane = (size_t)kTM * kKC * 2;
    const size_t abuf = ((3 * aplane + 1023) / 1024) * 1024;
    unsigned char* sB = sm;
    unsigned char* sA = sm + ((3 * bplane + 1023) / 1024) * 1024;   // [kStages] buffers
    uint64_t* full = reinterpret_cast<uint64_t*>(sA + kStages * abuf);   // [kStages]
    uint64_t* done = full + kStages;                                     // [kStages]
    uint64_t* dfull = done + kStages;                                    // [2]
    uint64_t* dempty = dfull + 2;                                        // [2]
    uint32_t* tslot = reinterpret_cast<uint32_t*>(dempty + 2);
    {   // B = Dw planes [3][nmpad][NIpad] staged K-major: rows = moments, K = directions
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
        for (int k = 0; k < kStages; ++k) {
            bar_init(&full[k], 256);
            bar_init(&done[k], 1);
        }
        for (int k = 0; k < 2; ++k) {
            bar_init(&dfull[k], 1);
            bar_init(&dempty[k], 128);
        }
    }
    if (warp == kD2mMma) tmem_alloc(tslot, 256);   // per tile buffer: leading-product and correction accumulators
    fence_async_smem();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tmem = *tslot;
    const int nchunks = NKpad / kKC;
    if (warp < kD2mEpi) {
        // ---- producers: set `set` takes the CTA's chunks c with c % kD2mSets == set ----
        const int set = warp >> 3;
        const int row = tid & 127, side = (tid >> 7) & 1;
        const long long my_tiles = (ntiles - 1 - (long long)blockIdx.x) / gridDim.x + 1;
        for (long long c = set; c < my_tiles * nchunks; c += kD2mSets) {
            const long long tile = blockIdx.x + (c / nchunks) * gridDim.x;
            const int ch = (int)(c % nchunks);
            const long long n = tile * kTM + row;
            const bool valid = n < NENK;
            const int s = (int)(c % kStages);
            const uint32_t u = (uint32_t)(c / kStages);
            float v[24];
            {
                const int i0 = ch * kKC + side * 24;
                const float* pp = psi + (size_t)i0 * (size_t)NENK + (valid ? n : 0);
                const int kn = valid ? NI - i0 : 0;   // directions of this half-chunk that exist
#pragma unroll
                for (int k = 0; k < 24; ++k) {
                    v[k] = k < kn ? __ldcs(pp) : 0.f;
                    pp += NENK;
                }
            }
            if (u > 0 && !bar_wait(&done[s], (u - 1) & 1u, err)) break;
            unsigned char* A = sA + s * abuf;
#pragma unroll
            for (int cl = 0; cl < 3; ++cl) {
                float w[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) w[k] = v[cl * 8 + k];
                uint4 hi, mid, lo;
                split8(w, hi, mid, lo);
                unsigned char* rp = A + (size_t)(side * 3 + cl) * kTM * 16 + (size_t)row * 16;
                *reinterpret_cast<uint4*>(rp) = hi;
                *reinterpret_cast<uint4*>(rp + aplane) = mid;
                *reinterpret_cast<uint4*>(rp + 2 * aplane) = lo;
            }
            fence_async_smem();
            bar_arrive(&full[s]);
        }
    } else if (warp < kD2mMma) {
        // ---- epilogue (TMEM lanes 32(w%4)..): out rows of the tile, 16 moments at a time ----
        const int r = tid - 32 * kD2mEpi;
        const uint32_t lane_base = tmem + ((uint32_t)((warp & 3) * 32) << 16);
        int it = 0;
        for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
            const int b = it & 1;
            const uint32_t u = (uint32_t)(it >> 1);
            const long long n = tile * kTM + r;
            const bool valid = n < NENK;
            double xv[16];
            const bool hx = xin && valid;
            const size_t nn = valid ? (size_t)n : 0;
            {
                const double* xp = hx ? xin + nn : nullptr;
#pragma unroll
                for (int k = 0; k < 16; ++k) {
                    xv[k] = (hx && k < nm) ? *xp : 0.0;
                    if (hx) xp += NENK;
                }
            }
            if (!bar_wait(&dfull[b], u & 1u, err)) break;
            tc_after_sync();
#pragma unroll
            for (int g = 0; g < KT; ++g) {
                // the leading product's accumulator plus the correction products' accumulator (IEEE FP32)
                float v[16], w[8];
                tmem_ld16(lane_base + (uint32_t)(b * 128 + g * 16), v);
                tmem_ld8(lane_base + (uint32_t)(b * 128 + 64 + g * 16), w);   // in halves: registers
#pragma unroll
                for (int k = 0; k < 8; ++k) v[k] += w[k];
                tmem_ld8(lane_base + (uint32_t)(b * 128 + 64 + g * 16 + 8), w);
#pragma unroll
                for (int k = 0; k < 8; ++k) v[8 + k] += w[k];
                if (valid) {
                    // one pointer stepped by a row per moment
                    double* op = out + (size_t)(g * 16) * (size_t)NENK + nn;
                    const int jn = nm - g * 16;
#pragma unroll
                    for (int k = 0; k < 16; ++k) {
                        if (k < jn) *op = beta * (double)v[k] + alpha * xv[k];
                        op += NENK;
                    }
                }
                // the next group's inputs
                if (g + 1 < KT) {
                    const double* xp = hx ? xin + (size_t)((g + 1) * 16) * (size_t)NENK + nn : nullptr;
                    const int jn = nm - (g + 1) * 16;
#pragma unroll
                    for (int k = 0; k < 16; ++k) {
                        xv[k] = (hx && k < jn) ? *xp : 0.0;
                        if (hx) xp += NENK;
                    }
                }
            }
            tc_before_sync();
            bar_arrive(&dempty[b]);
        }
    } else if ((tid & 31) == 0) {
        // ---- MMA issue ----
        const uint32_t idesc = idesc_bf16(kTM, nmpad);
        const uint32_t lboA = kTM * 16, lboB = (uint32_t)nmpad * 16;
        const uint32_t aBase = smem_u32(sA), bBase = smem_u32(sB);
        long long c = 0;
        int it = 0;
        bool ok = true;
        for (long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, ++it) {
            const int b = it & 1;
            const uint32_t ut = (uint32_t)(it >> 1);
            if (ut > 0 && !bar_wait(&dempty[b], (ut - 1) & 1u, err)) break;
            for (int ch = 0; ch < nchunks; ++ch, ++c) {
                const int s = (int)(c % kStages);
                const uint32_t u = (uint32_t)(c / kStages);
                if (!bar_wait(&full[s], u & 1u, err)) {
                    ok = false;
                    break;
                }
                tc_after_sync();
                const uint32_t a0 = aBase + s * (uint32_t)abuf;
                for (int ks = 0; ks < kKC / 16; ++ks)
                    for (int pr = 0; pr < 6; ++pr) {
                        const uint64_t da = sdesc(a0 + kProdA[pr] * (uint32_t)aplane + ks * 2 * lboA, lboA, 128);
                        const uint64_t db = sdesc(bBase + kProdB[pr] * (uint32_t)bplane +
                                                      (uint32_t)(ch * (kKC / 8) + ks * 2) * lboB, lboB, 128);
                        // product 5 (hi x hi) alone in columns b*128.., the five smaller ones in b*128 + 64..
                        const bool lead = pr == 5;
                        const uint32_t acc = lead ? (uint32_t)(ch | ks) : (uint32_t)(ch | ks | pr);
                        mma_bf16_ss(tmem + b * 128 + (lead ? 0u : 64u), da, db, idesc, acc ? 1u : 0u);
                    }
                mma_commit(&done[s]);
                if (ch == nchunks - 1) mma_commit(&dfull[b]);
            }
        }
    }
    tc_before_sync();
    __syncthreads();
    if (warp == kD2mMma) tmem_free(tmem, 256);
}

// ---------------------------------------------------------------------------------------------
// D2M with the angular vector streamed by the tensor-memory accelerator: the same product as
// d2m_tc_kernel, with psi brought into a ring of kT32 shared-memory stages by
// cp.async.bulk.tensor (a 2-D tensor map over psi[NI][NENK], box = 128 nodes x kKT directions;
// directions past NI and nodes past NENK are filled with zeros), so no thread waits on a global
// load.  Chunks of kKT = 32 directions (two MMA K-steps):
//   warp 0 lane 0    TMA issue: waits for a free FP32 stage, arms its barrier with the byte count and
//                    issues the copy;
//   warps 1-8        converters (kD2tSets sets of 8 warps taking alternate chunks; one set: 14 warps,
//                    at most 4 per SM sub-partition, so up to 128 registers a thread): threads t and
//                    t + 128 of a set take node t & 127 of the tile and 16 directions each, read them
//                    from the FP32 stage (then release it), split them into BF16 planes and write the
//                    A stage;
//   warps 9-12       epilogue, as d2m_tc_kernel (the warps index nodes by their TMEM lane quarter);
//   warp 13          lane 0 issues the MMAs; the warp owns the TMEM allocation.
// The leading split product (hi x hi) accumulates in its own TMEM accumulator and the five smaller
// products in a second one, added in the epilogue: the tensor core's accumulation of the full-size
// terms then runs over 18 MMAs per tile (288 directions) instead of all 108, which is where the split
// product lost accuracy against an FP32 GEMM (the small terms' accumulator is 2^-8 of the result).
// Every wait is bounded (error flag), as in the other kernels.  No cluster, no multicast.
// ---------------------------------------------------------------------------------------------
constexpr int kKT = 32;        // directions per K chunk
constexpr int kT32 = 5;        // FP32 stages (TMA ring)
constexpr int kTA = 2;         // BF16 A stages
constexpr int kD2tSets = 1;    // converter sets of 8 warps, taking alternate chunks
constexpr int kD2tConv = 1;    // first converter warp
constexpr int kD2tEpi = kD2tConv + 8 * kD2tSets;   // first epilogue warp
constexpr int kD2tMma = kD2tEpi + 4;               // the MMA warp
constexpr int kD2tThreads = 32 * (kD2tMma + 1);

// STACK: the three B planes are interleaved along N ([hi; mid; lo] rows per K column), so that one MMA of
// N = 3 nmpad takes hi x {hi, mid, lo}, one of N = 2 nmpad mid x {hi, mid} and one of N = nmpad lo x hi: each A
// plane is read from shared memory once per K step instead of once per product.  The accumulator of a tile
// holds three column groups (the hi x hi product, the 2^-8 products, the 2^-16 products), summed by the epilogue.
template <int KT, bool STACK>
__global__ void __launch_bounds__(kD2tThreads, 1) d2m_tma_kernel(const __grid_constant__ CUtensorMap psi_map,
                                                      const int* __restrict__ active,
                                                      const __nv_bfloat16* __restrict__ Dw, const double* xin,
                                                      double alpha, double beta, double* out, long long NENK, int NI,
                                                      int NIpad, int nm, int nmpad, long long ntiles, int* err) {
    if (active && *active == 0) return;
    extern __shared__ __align__(1024) unsigned char sm[];
    const int tid = threadIdx.x, warp = tid >> 5;
    const int NKpad = (NIpad + kKT - 1) / kKT * kKT;
    const size_t bplane = (size_t)nmpad * NKpad * 2;
    const size_t aplane = (size_t)kTM * kKT * 2;
    const size_t abuf = ((3 * aplane + 1023) / 1024) * 1024;
    constexpr size_t fbuf = (size_t)kTM * kKT * 4;                       // one FP32 stage
    unsigned char* sB = sm;
    unsigned char* sF = sm + ((3 * bplane + 1023) / 1024) * 1024;       // [kT32] FP32 stages
    unsigned char* sA = sF + kT32 * fbuf;                                // [kTA] A stages
    uint64_t* tfull = reinterpret_cast<uint64_t*>(sA + kTA * abuf);      // [kT32]
    uint64_t* tempty = tfull + kT32;                                     // [kT32]
    uint64_t* afull = tempty + kT32;                                     // [kTA]
    uint64_t* adone = afull + kTA;                                       // [kTA]
    uint64_t* dfull = adone + kTA;                                       // [2]
    uint64_t* dempty = dfull + 2;                                        // [2]
    uint32_t* tslot = reinterpret_cast<uint32_t*>(dempty + 2);
    {   // B = Dw planes [3][nmpad][NIpad] staged K-major: rows = moments, K = directions
        const int cc = NKpad / 8;
        const int total = 3 * nmpad * cc;
        for (int u = tid; u < total; u += blockDim.x) {
            const int p = u / (nmpad * cc);
            const int rem = u % (nmpad * cc);
            const int r = rem / cc, c = rem % cc;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (c * 8 < NIpad) v = __ldg(reinterpret_cast<const uint4*>(Dw + ((size_t)p * nmpad + r) * NIpad) + c);
            if (STACK)
                *reinterpret_cast<uint4*>(sB + (size_t)c * 3 * nmpad * 16 + (size_t)(p * nmpad + r) * 16) = v;
            else
                *reinterpret_cast<uint4*>(sB + p * bplane + (size_t)c * nmpad * 16 + (size_t)r * 16) = v;
        }
    }
    // TMEM columns per tile buffer: two groups of up to 64 (leading, corrections), or three of nmpad (STACK)
    constexpr uint32_t kBufCols = STACK ? 256u : 128u;
    if (tid == 0) {
        for (int k = 0; k < kT32; ++k) {
            bar_init(&tfull[k], 1);
            bar_init(&tempty[k], 256);
        }
        for (int k = 0; k < kTA; ++k) {
            bar_init(&afull[k], 256);
            bar_init(&adone[k], 1);
        }
        for (int k = 0; k < 2; ++k) {
            bar_init(&dfull[k], 1);
            bar_init(&dempty[k], 128);
        }
    }
    if (warp == kD2tMma) tmem_alloc(tslot, 2 * kBufCols);   // two tile buffers
    fence_async_smem();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tmem = *tslot;
    const int nchunks = NKpad / kKT;
    const long long my_tiles = (ntiles - 1 - (long long)blockIdx.x) / gridDim.x + 1;
    const long long nch = my_tiles * nchunks;
    if (warp == 0) {
        // ---- TMA issue ----
        if ((tid & 31) == 0) {
            for (long long c = 0; c < nch; ++c) {
                const int s = (int)(c % kT32);
                const uint32_t u = (uint32_t)(c / kT32);
                if (u > 0 && !bar_wait(&tempty[s], (u - 1) & 1u, err)) break;
                const long long tile = blockIdx.x + (c / nchunks) * gridDim.x;
                const int ch = (int)(c % nchunks);
                bar_expect_tx(&tfull[s], (uint32_t)fbuf);
                tma_load_2d(sF + s * fbuf, &psi_map, (int)(tile * kTM), ch * kKT, &tfull[s]);
            }
        }
    } else if (warp < kD2tEpi) {
        // ---- converters: FP32 stage -> BF16 planes of the A stage; set `set` takes chunks c = set mod kD2tSets ----
        const int t = tid - 32 * kD2tConv;
        const int row = t & 127, side = (t >> 7) & 1, set = t >> 8;
        for (long long c = set; c < nch; c += kD2tSets) {
            const int s = (int)(c % kT32);
            const int sa = (int)(c % kTA);
            if (!bar_wait(&tfull[s], (uint32_t)(c / kT32) & 1u, err)) break;
            const float* F = reinterpret_cast<const float*>(sF + s * fbuf) + (size_t)(side * 16) * kTM + row;
            float v[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) v[k] = F[(size_t)k * kTM];
            // the stage is refilled by the TMA (async proxy): order these generic reads before that write
            fence_async_smem();
            bar_arrive(&tempty[s]);
            const uint32_t ua = (uint32_t)(c / kTA);
            if (ua > 0 && !bar_wait(&adone[sa], (ua - 1) & 1u, err)) break;
            unsigned char* A = sA + sa * abuf;
#pragma unroll
            for (int cl = 0; cl < 2; ++cl) {
                float w[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) w[k] = v[cl * 8 + k];
                uint4 hi, mid, lo;
                split8(w, hi, mid, lo);
                unsigned char* rp = A + (size_t)(side * 2 + cl) * kTM * 16 + (size_t)row * 16;
                *reinterpret_cast<uint4*>(rp) = hi;
                *reinterpret_cast<uint4*>(rp + aplane) = mid;
                *reinterpret_cast<uint4*>(rp + 2 * aplane) = lo;
            }
            fence_async_smem();
            bar_arrive(&afull[sa]);
        }
    } else if (warp < kD2tMma) {
        // ---- epilogue: a warp reads TMEM lanes 32(w%4).. (the hardware's lane quarter of warp w), i.e.
        // tile nodes 32(w%4) + lane ----
        const int r = ((warp & 3) << 5) | (tid & 31);
        const uint32_t lane_base = tmem + ((uint32_t)((warp & 3) * 32) << 16);
        int it = 0;
        for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
            const int b = it & 1;
            const uint32_t u = (uint32_t)(it >> 1);
            const long long n = tile * kTM + r;
            const bool valid = n < NENK;
            double xv[16];
            const bool hx = xin && valid;
            const size_t nn = valid ? (size_t)n : 0;
            {
                const double* xp = hx ? xin + nn : nullptr;
#pragma unroll
                for (int k = 0; k < 16; ++k) {
                    xv[k] = (hx && k < nm) ? *xp : 0.0;
                    if (hx) xp += NENK;
                }
            }
            if (!bar_wait(&dfull[b], u & 1u, err)) break;
            tc_after_sync();
#pragma unroll
            for (int g = 0; g < KT; ++g) {
                // the leading product's accumulator plus the correction products' accumulator(s) (IEEE FP32)
                float v[16], w[16];
                if (STACK) {
                    tmem_ld16(lane_base + (uint32_t)(b * kBufCols + nmpad + g * 16), w);
                    tmem_ld16(lane_base + (uint32_t)(b * kBufCols + 2 * nmpad + g * 16), v);
#pragma unroll
                    for (int k = 0; k < 16; ++k) w[k] += v[k];
                    tmem_ld16(lane_base + (uint32_t)(b * kBufCols + g * 16), v);
                } else {
                    tmem_ld16(lane_base + (uint32_t)(b * kBufCols + g * 16), v);
                    tmem_ld16(lane_base + (uint32_t)(b * kBufCols + 64 + g * 16), w);
                }
#pragma unroll
                for (int k = 0; k < 16; ++k) v[k] += w[k];
                if (valid) {
                    double* op = out + (size_t)(g * 16) * (size_t)NENK + nn;
                    const int jn = nm - g * 16;
#pragma unroll
                    for (int k = 0; k < 16; ++k) {
                        if (k < jn) *op = beta * (double)v[k] + alpha * xv[k];
                        op += NENK;
                    }
                }
                if (g + 1 < KT) {
                    const double* xp = hx ? xin + (size_t)((g + 1) * 16) * (size_t)NENK + nn : nullptr;
                    const int jn = nm - (g + 1) * 16;
#pragma unroll
                    for (int k = 0; k < 16; ++k) {
                        xv[k] = (hx && k < jn) ? *xp : 0.0;
                        if (hx) xp += NENK;
                    }
                }
            }
            tc_before_sync();
            bar_arrive(&dempty[b]);
        }
    } else if ((tid & 31) == 0) {
        // ---- MMA issue ----
        const uint32_t idesc = idesc_bf16(kTM, nmpad);
        const uint32_t lboA = kTM * 16, lboB = (uint32_t)nmpad * 16 * (STACK ? 3u : 1u);
        const uint32_t aBase = smem_u32(sA), bBase = smem_u32(sB);
        long long c = 0;
        int it = 0;
        bool ok = true;
        for (long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, ++it) {
            const int b = it & 1;
            const uint32_t ut = (uint32_t)(it >> 1);
            if (ut > 0 && !bar_wait(&dempty[b], (ut - 1) & 1u, err)) break;
            for (int ch = 0; ch < nchunks; ++ch, ++c) {
                const int sa = (int)(c % kTA);
                if (!bar_wait(&afull[sa], (uint32_t)(c / kTA) & 1u, err)) {
                    ok = false;
                    break;
                }
                tc_after_sync();
                const uint32_t a0 = aBase + sa * (uint32_t)abuf;
                if (STACK) {
                    // hi x [hi; mid; lo] -> groups 0, 1, 2; mid x [hi; mid] -> groups 1, 2; lo x hi -> group 2
                    const uint32_t d0 = tmem + (uint32_t)b * kBufCols;
                    for (int ks = 0; ks < kKT / 16; ++ks) {
                        const uint64_t db = sdesc(bBase + (uint32_t)(ch * (kKT / 8) + ks * 2) * lboB, lboB, 128);
                        const uint32_t ka = a0 + ks * 2 * lboA;
                        mma_bf16_ss(d0, sdesc(ka, lboA, 128), db, idesc_bf16(kTM, 3 * nmpad), (ch | ks) ? 1u : 0u);
                        mma_bf16_ss(d0 + nmpad, sdesc(ka + (uint32_t)aplane, lboA, 128), db, idesc_bf16(kTM, 2 * nmpad),
                                    1u);
                        mma_bf16_ss(d0 + 2 * nmpad, sdesc(ka + 2 * (uint32_t)aplane, lboA, 128), db, idesc, 1u);
                    }
                } else {
                    for (int ks = 0; ks < kKT / 16; ++ks)
                        for (int pr = 0; pr < 6; ++pr) {
                            const uint64_t da = sdesc(a0 + kProdA[pr] * (uint32_t)aplane + ks * 2 * lboA, lboA, 128);
                            const uint64_t db = sdesc(bBase + kProdB[pr] * (uint32_t)bplane +
                                                          (uint32_t)(ch * (kKT / 8) + ks * 2) * lboB, lboB, 128);
                            // product 5 (hi x hi) alone in columns b*128.., the five smaller ones in b*128 + 64..
                            const bool lead = pr == 5;
                            const uint32_t acc = lead ? (uint32_t)(ch | ks) : (uint32_t)(ch | ks | pr);
                            mma_bf16_ss(tmem + b * kBufCols + (lead ? 0u : 64u), da, db, idesc, acc ? 1u : 0u);
                        }
                }
                mma_commit(&adone[sa]);
                if (ch == nchunks - 1) mma_commit(&dfull[b]);
            }
        }
    }
    tc_before_sync();
    __syncthreads();
    if (warp == kD2tMma) tmem_free(tmem, 2 * kBufCols);
}

size_t d2m_tma_smem(int NIpad, int nmpad) {
    const int NKpad = (NIpad + kKT - 1) / kKT * kKT;
    const size_t b = ((3 * (size_t)nmpad * NKpad * 2 + 1023) / 1024) * 1024;
    const size_t a = ((3 * (size_t)kTM * kKT * 2 + 1023) / 1024) * 1024;
    return b + kT32 * (size_t)kTM * kKT * 4 + kTA * a + 8 * (2 * kT32 + 2 * kTA + 4) + 16;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against libcuda).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

size_t m2d_tc_smem(int NH, int nmpad, int mode = 0, int nm = 0) {
    const size_t b = ((3 * (size_t)NH * nmpad * 2 + 1023) / 1024) * 1024;
    const size_t a = ((3 * (size_t)kTM * nmpad * 2 + 1023) / 1024) * 1024;
    if (mode == 0) return b + 2 * a + 96;
    if (mode == 1) return b + 2 * a + 1024 + (size_t)kM2dEpi * 2 * 2048;
    return b + 2 * a + 1024 + (size_t)kM2dEpi * 2048 + 2 * (size_t)kTM * nm * 8;
}

size_t d2m_tc_smem(int NIpad, int nmpad) {
    const int NKpad = (NIpad + kKC - 1) / kKC * kKC;
    const size_t b = ((3 * (size_t)nmpad * NKpad * 2 + 1023) / 1024) * 1024;
    const size_t a = ((3 * (size_t)kTM * kKC * 2 + 1023) / 1024) * 1024;
    return b + kStages * a + 128;
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

// The TMA-fed D2M (LB_MOMENTS_TMA=0: the register-fed kernel).
bool moments_tma_enabled() {
    static int on = -1;
    if (on < 0) {
        const char* e = std::getenv("LB_MOMENTS_TMA");
        on = (e && *e == '0') ? 0 : 1;
    }
    return on == 1;
}

// D2M's B planes stacked along N, three MMAs per K step (LB_D2M_STACK=0: six MMAs, one per product).
bool d2m_stack_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("LB_D2M_STACK");
        return !(e && *e == '0');
    }();
    return on;
}

// M2D's output written by TMA stores (LB_M2D_TMA_STORE=0: per-thread stores).
bool moments_tma_store_enabled() {
    static int on = -1;
    if (on < 0) {
        const char* e = std::getenv("LB_M2D_TMA_STORE");
        on = (e && *e == '0') ? 0 : 1;
    }
    return on == 1;
}

// M2D's moment tiles loaded by TMA (LB_M2D_TMA_LOAD=0: per-thread loads).
bool moments_tma_load_enabled() {
    static int on = -1;
    if (on < 0) {
        const char* e = std::getenv("LB_M2D_TMA_LOAD");
        on = (e && *e == '0') ? 0 : 1;
    }
    return on == 1;
}

// Returns LB_ERR_ARG when the shape does not fit the tensor-core kernels (caller falls back).
int launch_m2d_tc(Handle* h, const double* x, const float* sigl, const double* a, const float* qadd, float* q) {
    const int nhalves = h->NIpad > 256 ? 2 : 1;
    const int NH = ((h->NIpad + nhalves - 1) / nhalves + 15) / 16 * 16;
    if (NH > 256 || h->nmpad % 16 || h->nmpad > 64 || h->NIpad % 8) return LB_ERR_ARG;
    // one CTA per SM (it holds all 512 TMEM columns: two accumulators of up to 256)
    int* err = h->d_tc_err;
    if (!err) return LB_ERR_STATE;
    // TMA stores of the output when there is no added source and a tensor map can be made
    CUtensorMap map;
    std::memset(&map, 0, sizeof(map));
    CUtensorMap xmap;
    std::memset(&xmap, 0, sizeof(xmap));
    EncodeTiledFn enc = encode_tiled();
    bool ts = enc && !qadd && moments_tma_store_enabled() && m2d_tc_smem(NH, h->nmpad, 1) <= 227 * 1024 &&
              !((uintptr_t)q & 15) && h->NENK < (1LL << 31);
    if (ts) {
        const cuuint64_t dims[2] = {(cuuint64_t)h->NENK, (cuuint64_t)h->NI};
        const cuuint64_t strides[1] = {(cuuint64_t)h->NENK * 4};
        const cuuint32_t box[2] = {32u, 16u};
        const cuuint32_t estr[2] = {1, 1};
        ts = enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, q, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                 CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
    }
    // the moment tiles by TMA as well, from whichever operand holds them (x, or the add operand when x is
    // null: the group sources), not when both are given; the two stages must fit
    const double* src = x ? x : a;
    bool tl = ts && src && !(x && a) && moments_tma_load_enabled() && h->nm <= 256 &&
              m2d_tc_smem(NH, h->nmpad, 2, h->nm) <= 227 * 1024 && !((uintptr_t)src & 15);
    if (tl) {
        const cuuint64_t dims[2] = {(cuuint64_t)h->NENK, (cuuint64_t)h->nm};
        const cuuint64_t strides[1] = {(cuuint64_t)h->NENK * 8};
        const cuuint32_t box[2] = {(cuuint32_t)kTM, (cuuint32_t)h->nm};
        const cuuint32_t estr[2] = {1, 1};
        tl = enc(&xmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(src), dims, strides, box, estr,
                 CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
    }
    const int mode = tl ? 2 : ts ? 1 : 0;
    const size_t smem = std::max<size_t>(m2d_tc_smem(NH, h->nmpad, mode, h->nm), 116 * 1024);
    if (smem > 227 * 1024) return LB_ERR_ARG;
    static PerDevice attr;
    attr.get([&] {
#define LB_M2DATTR(K)                                                                                      \
    cudaFuncSetAttribute(m2d_tc_kernel<K, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);   \
    cudaFuncSetAttribute(m2d_tc_kernel<K, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);   \
    cudaFuncSetAttribute(m2d_tc_kernel<K, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024)
        LB_M2DATTR(1);
        LB_M2DATTR(2);
        LB_M2DATTR(3);
        LB_M2DATTR(4);
#undef LB_M2DATTR
        return 1;
    });
    const long long ntiles = (h->NENK + kTM - 1) / kTM;
    long long grid = std::min<long long>(ntiles * nhalves, (long long)h->sm_count);
    grid = std::max<long long>(nhalves, grid / nhalves * nhalves);
#define LB_M2DTC(K, M)                                                                                              \
    m2d_tc_kernel<K, M><<<(int)grid, M == 2 ? kM2dThreadsTma : kM2dThreads, smem, h->stream>>>(                      \
        map, xmap, h->d_active, x, sigl, a, qadd, h->d_mat, h->d_Ym2d, q, h->NENK, h->NI, h->NIpad, h->nm, h->nmpad, \
        NH, nhalves, ntiles, err)
#define LB_M2DK(K)                           \
    if (mode == 2) LB_M2DTC(K, 2);           \
    else if (mode == 1) LB_M2DTC(K, 1);      \
    else LB_M2DTC(K, 0)
    switch (h->nmpad / 16) {
        case 1: LB_M2DK(1); break;
        case 2: LB_M2DK(2); break;
        case 3: LB_M2DK(3); break;
        default: LB_M2DK(4); break;
    }
#undef LB_M2DK
#undef LB_M2DTC
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LB_OK : cuda_fail(h, e, "m2d tensor-core kernel");
}

// The TMA-fed D2M; LB_ERR_ARG when it does not apply (no tensor-map encoder, shape, alignment).
int launch_d2m_tma(Handle* h, const float* psi, const double* xin, double alpha, double beta, double* out) {
    EncodeTiledFn enc = encode_tiled();
    if (!enc || !moments_tma_enabled()) return LB_ERR_ARG;
    if (h->nmpad > 64 || h->nmpad % 16 || h->NIpad % 8 || ((uintptr_t)psi & 15) || (h->NENK * 4) % 16 ||
        h->NENK >= (1LL << 31) || h->NI < 1)
        return LB_ERR_ARG;
    const size_t smem = std::max<size_t>(d2m_tma_smem(h->NIpad, h->nmpad), 116 * 1024);
    if (smem > 227 * 1024) return LB_ERR_ARG;
    int* err = h->d_tc_err;
    if (!err) return LB_ERR_STATE;
    // tensor map over psi[NI][NENK] (FP32): box 128 nodes x kKT directions, zero fill outside
    CUtensorMap map;
    const cuuint64_t dims[2] = {(cuuint64_t)h->NENK, (cuuint64_t)h->NI};
    const cuuint64_t strides[1] = {(cuuint64_t)h->NENK * 4};
    const cuuint32_t box[2] = {(cuuint32_t)kTM, (cuuint32_t)kKT};
    const cuuint32_t estr[2] = {1, 1};
    if (enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(psi), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return LB_ERR_ARG;
    static PerDevice attr;
    attr.get([&] {
#define LB_D2MATTR(K, S) cudaFuncSetAttribute(d2m_tma_kernel<K, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024)
        LB_D2MATTR(1, false); LB_D2MATTR(2, false); LB_D2MATTR(3, false); LB_D2MATTR(4, false);
        LB_D2MATTR(1, true); LB_D2MATTR(2, true); LB_D2MATTR(3, true); LB_D2MATTR(4, true);
#undef LB_D2MATTR
        return 1;
    });
    const long long ntiles = (h->NENK + kTM - 1) / kTM;
    const long long grid = std::min<long long>(ntiles, (long long)h->sm_count);
    const bool stack = d2m_stack_enabled();
#define LB_D2MTMA(K)                                                                                                    \
    if (stack)                                                                                                          \
        d2m_tma_kernel<K, true><<<(int)grid, kD2tThreads, smem, h->stream>>>(map, h->d_active, h->d_Yd2m, xin, alpha,   \
                                                                           beta, out, h->NENK, h->NI, h->NIpad, h->nm, \
                                                                           h->nmpad, ntiles, err);                     \
    else                                                                                                                \
        d2m_tma_kernel<K, false><<<(int)grid, kD2tThreads, smem, h->stream>>>(map, h->d_active, h->d_Yd2m, xin, alpha,  \
                                                                            beta, out, h->NENK, h->NI, h->NIpad, h->nm, \
                                                                            h->nmpad, ntiles, err)
    switch (h->nmpad / 16) {
        case 1: LB_D2MTMA(1); break;
        case 2: LB_D2MTMA(2); break;
        case 3: LB_D2MTMA(3); break;
        default: LB_D2MTMA(4); break;
    }
#undef LB_D2MTMA
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LB_OK : cuda_fail(h, e, "d2m TMA kernel");
}

int launch_d2m_tc(Handle* h, const float* psi, const double* xin, double alpha, double beta, double* out) {
    {
        const int rc = launch_d2m_tma(h, psi, xin, alpha, beta, out);
        if (rc != LB_ERR_ARG) return rc;
    }
    if (h->nmpad > 64 || h->nmpad % 16 || h->NIpad % 8) return LB_ERR_ARG;
    // one CTA per SM (two accumulators of up to 64 columns in a 128-column allocation)
    const size_t smem = std::max<size_t>(d2m_tc_smem(h->NIpad, h->nmpad), 116 * 1024);
    if (smem > 227 * 1024) return LB_ERR_ARG;
    int* err = h->d_tc_err;
    if (!err) return LB_ERR_STATE;
    static PerDevice attr;
    attr.get([&] {
        cudaFuncSetAttribute(d2m_tc_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        cudaFuncSetAttribute(d2m_tc_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        cudaFuncSetAttribute(d2m_tc_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        cudaFuncSetAttribute(d2m_tc_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        return 1;
    });
    const long long ntiles = (h->NENK + kTM - 1) / kTM;
    const long long grid = std::min<long long>(ntiles, (long long)h->sm_count);
#define LB_D2MTC(K)                                                                                         \
    d2m_tc_kernel<K><<<(int)grid, kD2mThreads, smem, h->stream>>>(h->d_active, psi, h->d_Yd2m, xin, alpha, beta, out, \
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

namespace {
// One thread waits on a pipeline barrier that nothing arrives at, with the contraction kernels' bounded wait
// cut to `limit` polls: it gives up, raises the handle's error flag and returns, as a stuck stage would.
__global__ void tc_wait_probe_kernel(int* err, long long limit) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        bar_init(&bar, 1);
        bar_wait(&bar, 0u, err, limit);
    }
}
}  // namespace

int tc_wait_probe(Handle* h, long long polls) {
    if (!h->d_tc_err) return LB_ERR_STATE;
    tc_wait_probe_kernel<<<1, 32, 0, h->stream>>>(h->d_tc_err, polls);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(h, e, "wait probe launch");
    return moments_tc_status(h);
}

// Reads and clears the handle's contraction timeout flag (synchronises the handle's stream): LB_ERR_TIMEOUT
// when a tensor-core contraction gave up on a pipeline wait since the last check.
int moments_tc_status(Handle* h) {
    if (!h->d_tc_err) return LB_OK;
    int v = 0;
    cudaError_t e = cudaMemcpyAsync(&v, h->d_tc_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "contraction status");
    if (!v) return LB_OK;
    e = cudaMemsetAsync(h->d_tc_err, 0, sizeof(int), h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "contraction status");
    return fail(h, LB_ERR_TIMEOUT, "tensor-core moment kernel: pipeline wait timed out (results invalid)");
}

}  // namespace lb
