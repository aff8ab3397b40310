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
// The schedules share that element update:
//  * cluster levels: blocks of 6 consecutive elements (a hex of a box mesh split into 6 tets) are
//    swept as units over each direction's block-level graph, one thread per block, a CTA barrier
//    between block levels; optionally with the element matrices of every element type computed once
//    per direction.  The fastest at the 768k-tet configuration.
//  * levels: one CTA owns whole directions and walks their element wavefront levels in order with a
//    CTA barrier between levels; upstream values written by the same SM are re-read through its L1.
//  * levels with next-level prefetch, element flags in shared memory, grouped same-schedule
//    directions, and dataflow (warps claim 32-element chunks from a global counter and wait, with a
//    bounded spin, on the completion counter of the previous level): candidates for other meshes.
// Launch shape (schedule, threads per CTA, directions or CTAs per SM, updates in flight per thread)
// is picked by timing the first sweeps of a handle (the three fastest twice); every candidate
// computes bit-identical results.
#include "lb_internal.h"
#include <algorithm>
#include <cstdio>
#include <cstdlib>

namespace lb {

namespace {

constexpr float kThird = 1.0f / 3.0f;
constexpr float kFiveThirds = 5.0f / 3.0f;
constexpr float kFourThirds = 4.0f / 3.0f;
// Padding entry of the padded sweep order.  Real items can be negative (bit 31 carries the outflow
// flag of face 3), so padding is recognised by equality; no real item is all ones because element
// ids stay below 0xFFFFFF.
constexpr int kPad = -1;

struct SweepArgs {
    const int* __restrict__ items;
    const int* __restrict__ pitems;
    const long long* __restrict__ pbase;
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
    const int4* __restrict__ rec;     // 16-byte element records with type indices (when ngeom > 0)
    const float4* __restrict__ gtab;  // [ngeom][3] face vectors of the element types
    const int* __restrict__ tmat;     // [ngeom] material of the element types
    int ngeom;
    const int4* __restrict__ crec;    // block records (cluster schedule), direction i's from crec_base[i]
    const long long* __restrict__ crec_base;
    const int* __restrict__ blk_elem; // [nclusters][kClusterSize] block members, or null: consecutive ids
    const int* __restrict__ cl_start;
    const int* __restrict__ cl_base;
    const int* __restrict__ ncl;
    int nclusters;                    // 0: no cluster schedule
};

__device__ __forceinline__ float pick(const float4& v, int idx) {
    float r = v.x;
    r = (idx == 1) ? v.y : r;
    r = (idx == 2) ? v.z : r;
    r = (idx == 3) ? v.w : r;
    return r;
}

__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
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
struct Geom {
    float4 gx, gy, gz;
    int4 gn;
};

// The 64-byte element record is read with two 256-bit loads (32-byte aligned): half the load
// instructions and L1 sector accesses of four 128-bit loads.
__device__ __forceinline__ void ld_nc_v8(const float* p, float (&r)[8]) {
    asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=f"(r[0]), "=f"(r[1]), "=f"(r[2]), "=f"(r[3]), "=f"(r[4]), "=f"(r[5]), "=f"(r[6]), "=f"(r[7])
        : "l"(p));
}

__device__ __forceinline__ Geom load_geom(const float4* __restrict__ geom, int e) {
    const float* p = reinterpret_cast<const float*>(geom + (size_t)e * 4);
    float a[8], b[8];
    ld_nc_v8(p, a);
    ld_nc_v8(p + 8, b);
    Geom g;
    g.gx = make_float4(a[0], a[1], a[2], a[3]);
    g.gy = make_float4(a[4], a[5], a[6], a[7]);
    g.gz = make_float4(b[0], b[1], b[2], b[3]);
    g.gn = make_int4(__float_as_int(b[4]), __float_as_int(b[5]), __float_as_int(b[6]), __float_as_int(b[7]));
    return g;
}

template <bool kCG, bool kHaveQ = false, int kPrev = 0>
__device__ __forceinline__ void assemble_g(const float* base, float4 dir, int item, const Geom& G, const float* s_sigt,
                                           Update& u, float4 qpre, int prev_e = -1,
                                           float4 prev_v = make_float4(0.f, 0.f, 0.f, 0.f), int prev2_e = -1,
                                           float4 prev2_v = make_float4(0.f, 0.f, 0.f, 0.f));

// Element from its 16-byte record (one 128-bit load) and the type table in shared memory.  The type
// index sits in the bits that otherwise carry the material, so the element update reads it as the
// material id and the CTA's cross-section table is indexed by type (load_gtab).
__device__ __forceinline__ Geom geom_from_rec(int4 rec, const float4* s_gtab) {
    Geom g;
    g.gn = rec;
    const int t = (int)(((unsigned)g.gn.x >> 30) | (((unsigned)g.gn.y >> 30) << 2) | (((unsigned)g.gn.z >> 30) << 4) |
                        (((unsigned)g.gn.w >> 30) << 6));
    g.gx = s_gtab[3 * t + 0];
    g.gy = s_gtab[3 * t + 1];
    g.gz = s_gtab[3 * t + 2];
    return g;
}

__device__ __forceinline__ Geom load_geom_tab(const int4* __restrict__ rec, const float4* s_gtab, int e) {
    return geom_from_rec(__ldg(&rec[e]), s_gtab);
}

// Copies the type table into shared memory (kernels launched with 48 * ngeom bytes of dynamic shared
// memory) and re-indexes the cross sections by type; returns the table, or nullptr when the mesh has
// none (then s_sigt stays indexed by material).
__device__ __forceinline__ const float4* load_gtab(const SweepArgs& a, float4* s_gtab, float* s_sigt) {
    if (a.ngeom <= 0) return nullptr;
    __syncthreads();   // s_sigt was filled by material
    float st = 0.f;
    if (threadIdx.x < a.ngeom) st = a.sigt[__ldg(&a.tmat[threadIdx.x])];
    for (int k = threadIdx.x; k < 3 * a.ngeom; k += blockDim.x) s_gtab[k] = __ldg(&a.gtab[k]);
    __syncthreads();
    if (threadIdx.x < 256) s_sigt[threadIdx.x] = threadIdx.x < a.ngeom ? st : 0.f;
    __syncthreads();
    return s_gtab;
}

template <bool kCG, bool kHaveQ = false>
__device__ __forceinline__ void assemble(const SweepArgs& a, const float* base, float4 dir, int item,
                                         const float* s_sigt, Update& u, float4 qpre = make_float4(0.f, 0.f, 0.f, 0.f),
                                         const float4* s_gtab = nullptr) {
    const Geom G = s_gtab ? load_geom_tab(a.rec, s_gtab, item & 0xFFFFFF) : load_geom(a.geom, item & 0xFFFFFF);
    assemble_g<kCG, kHaveQ>(base, dir, item, G, s_sigt, u, qpre);
}

// kPrev >= 1: the solution of element prev_e (the thread's previous update) is passed in registers and used
// instead of a load when it is an upstream neighbour; kPrev = 2 also the one before it (prev2_e).
template <bool kCG, bool kHaveQ, int kPrev>
__device__ __forceinline__ void assemble_g(const float* base, float4 dir, int item, const Geom& G, const float* s_sigt,
                                           Update& u, float4 qpre, int prev_e, float4 prev_v, int prev2_e,
                                           float4 prev2_v) {
    // gmsh face -> local nodes; the vertex opposite face f is 3 - f
    constexpr int F[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
    const int e = item & 0xFFFFFF;
    const int upm = (item >> 24) & 0xF;
    const int outm = (item >> 28) & 0xF;
    const float4 gx = G.gx, gy = G.gy, gz = G.gz;
    const int4 gn = G.gn;
    const float4 q = kHaveQ ? qpre : ld4<kCG>(base + 4 * (size_t)e);
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
            const float4 u4 = (kPrev >= 1 && ep == prev_e)   ? prev_v
                              : (kPrev >= 2 && ep == prev2_e) ? prev2_v
                                                              : ld4<kCG>(base + 4 * (size_t)ep);
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
    const float idet = __fdividef(1.0f, det);
    const float z0 = fmaf(e11, v0, -4.0f * v1) * idet;
    const float z1 = fmaf(e00, v1, -ba * v0) * idet;
    const float id = __fdividef(1.0f, u.d);
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

// Per-type element table of one direction (meshes with an element type table).  The element matrix
// T = d I + a 1^T + 1 b^T and the factors of its 2x2 capacitance solve depend only on the element's
// shape and material (its type), the direction and the outflow-face mask, so a CTA computes them
// once per type when it starts a direction -- with the same operations as assemble_g and
// solve_rank2, hence bit-identical -- and an update only adds the upstream terms and applies the
// factors.  The table is built for the outflow mask given by the signs of the FP32 face
// coefficients; an element whose schedule item carries another mask (the FP64 test in the
// schedule can differ for a face nearly parallel to the direction) takes the full path.
struct ElemTab {
    float4 c;    // c_f = k . s_f
    float4 a;    // a_k
    float4 b;    // b_k
    float4 s0;   // e00, e11, b.a, 1 / det
    float4 s1;   // 1 / d, outflow mask (int bits), -, -
};

__device__ __forceinline__ void build_tab(const float4* s_gtab, const float* s_sigt, int ngeom, float4 dir,
                                          ElemTab* s_tab) {
    for (int t = threadIdx.x; t < ngeom; t += blockDim.x) {
        const float4 gx = s_gtab[3 * t + 0], gy = s_gtab[3 * t + 1], gz = s_gtab[3 * t + 2];
        float c[4];
        c[0] = fmaf(dir.x, gx.x, fmaf(dir.y, gy.x, dir.z * gz.x));
        c[1] = fmaf(dir.x, gx.y, fmaf(dir.y, gy.y, dir.z * gz.y));
        c[2] = fmaf(dir.x, gx.z, fmaf(dir.y, gy.z, dir.z * gz.z));
        c[3] = fmaf(dir.x, gx.w, fmaf(dir.y, gy.w, dir.z * gz.w));
        int outm = 0;
#pragma unroll
        for (int f = 0; f < 4; ++f) outm |= (c[f] < 0.0f) ? 0 : (1 << f);
        Update u;
        float co[4];
#pragma unroll
        for (int f = 0; f < 4; ++f) co[f] = ((outm >> f) & 1) ? c[f] : 0.0f;
        const float Ct = (co[0] + co[1]) + (co[2] + co[3]);
        u.d = fmaf(kFiveThirds, Ct, s_sigt[t]);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            u.a[k] = kFiveThirds * (c[3 - k] - co[3 - k]);
            u.b[k] = (Ct - co[3 - k]) * kThird;
        }
        const float sa = (u.a[0] + u.a[1]) + (u.a[2] + u.a[3]);
        const float sb = (u.b[0] + u.b[1]) + (u.b[2] + u.b[3]);
        const float ba = fmaf(u.b[0], u.a[0], fmaf(u.b[1], u.a[1], fmaf(u.b[2], u.a[2], u.b[3] * u.a[3])));
        const float e00 = u.d + sa, e11 = u.d + sb;
        const float det = fmaf(e00, e11, -4.0f * ba);
        ElemTab T;
        T.c = make_float4(c[0], c[1], c[2], c[3]);
        T.a = make_float4(u.a[0], u.a[1], u.a[2], u.a[3]);
        T.b = make_float4(u.b[0], u.b[1], u.b[2], u.b[3]);
        T.s0 = make_float4(e00, e11, ba, __fdividef(1.0f, det));
        T.s1 = make_float4(__fdividef(1.0f, u.d), __int_as_float(outm), 0.f, 0.f);
        s_tab[t] = T;
    }
}

// One element update through the direction's type table (falls back to assemble + finish).
template <bool kCG>
__device__ __forceinline__ void update_tab(const SweepArgs& a, float* base, float4 dir, int item, const float* s_sigt,
                                           const float4* s_gtab, const ElemTab* s_tab) {
    constexpr int F[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
    const int e = item & 0xFFFFFF;
    const int upm = (item >> 24) & 0xF;
    const int outm = (item >> 28) & 0xF;
    const int4 gn = __ldg(&a.rec[e]);
    const unsigned nw[4] = {(unsigned)gn.x, (unsigned)gn.y, (unsigned)gn.z, (unsigned)gn.w};
    const int t = (int)((nw[0] >> 30) | ((nw[1] >> 30) << 2) | ((nw[2] >> 30) << 4) | ((nw[3] >> 30) << 6));
    const ElemTab* T = s_tab + t;
    if (outm != __float_as_int(T->s1.y)) {
        Update u;
        assemble_g<kCG>(base, dir, item, geom_from_rec(gn, s_gtab), s_sigt, u, make_float4(0.f, 0.f, 0.f, 0.f));
        finish<kCG>(base, item, u);
        return;
    }
    const float4 q = ld4<kCG>(base + 4 * (size_t)e);
    const float4 c4 = T->c;
    const float c[4] = {c4.x, c4.y, c4.z, c4.w};
    float r[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        if ((upm >> f) & 1) {
            const unsigned wd = nw[f];
            const float4 u4 = ld4<kCG>(base + 4 * (size_t)(wd & 0xFFFFFFu));
            const float u0 = pick(u4, (wd >> 24) & 3);
            const float u1 = pick(u4, (wd >> 26) & 3);
            const float u2 = pick(u4, (wd >> 28) & 3);
            const float U = u0 + u1 + u2;
            const float cf = c[f];
            const float t3 = U * kThird;
            r[F[f][0]] = fmaf(-cf, fmaf(kFiveThirds, u0, t3), r[F[f][0]]);
            r[F[f][1]] = fmaf(-cf, fmaf(kFiveThirds, u1, t3), r[F[f][1]]);
            r[F[f][2]] = fmaf(-cf, fmaf(kFiveThirds, u2, t3), r[F[f][2]]);
            r[3 - f] = fmaf(cf * kFourThirds, U, r[3 - f]);
        }
    }
    const float4 A = T->a, B = T->b, S0 = T->s0;
    const float id = T->s1.x;
    const float v0 = (r[0] + r[1]) + (r[2] + r[3]);
    const float v1 = fmaf(B.x, r[0], fmaf(B.y, r[1], fmaf(B.z, r[2], B.w * r[3])));
    const float z0 = fmaf(S0.y, v0, -4.0f * v1) * S0.w;
    const float z1 = fmaf(S0.x, v1, -S0.z * v0) * S0.w;
    const float4 v = make_float4((r[0] - fmaf(A.x, z0, z1)) * id, (r[1] - fmaf(A.y, z0, z1)) * id,
                                 (r[2] - fmaf(A.z, z0, z1)) * id, (r[3] - fmaf(A.w, z0, z1)) * id);
    if (kCG) __stcg(reinterpret_cast<float4*>(base + 4 * (size_t)e), v);
    else *reinterpret_cast<float4*>(base + 4 * (size_t)e) = v;
}

// update_tab with the element's 16-byte record and its source already loaded (the cluster kernel
// fetches both for the next element of a block while it updates the current one).
template <bool kCG>
__device__ __forceinline__ void update_tab_pre(const SweepArgs& a, float* base, float4 dir, int item, int4 gn, float4 q,
                                               const float* s_sigt, const float4* s_gtab, const ElemTab* s_tab) {
    constexpr int F[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
    const int e = item & 0xFFFFFF;
    const int upm = (item >> 24) & 0xF;
    const int outm = (item >> 28) & 0xF;
    const unsigned nw[4] = {(unsigned)gn.x, (unsigned)gn.y, (unsigned)gn.z, (unsigned)gn.w};
    const int t = (int)((nw[0] >> 30) | ((nw[1] >> 30) << 2) | ((nw[2] >> 30) << 4) | ((nw[3] >> 30) << 6));
    const ElemTab* T = s_tab + t;
    if (outm != __float_as_int(T->s1.y)) {
        Update u;
        assemble_g<kCG, true>(base, dir, item, geom_from_rec(gn, s_gtab), s_sigt, u, q);
        finish<kCG>(base, item, u);
        return;
    }
    const float4 c4 = T->c;
    const float c[4] = {c4.x, c4.y, c4.z, c4.w};
    float r[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        if ((upm >> f) & 1) {
            const unsigned wd = nw[f];
            const float4 u4 = ld4<kCG>(base + 4 * (size_t)(wd & 0xFFFFFFu));
            const float u0 = pick(u4, (wd >> 24) & 3);
            const float u1 = pick(u4, (wd >> 26) & 3);
            const float u2 = pick(u4, (wd >> 28) & 3);
            const float U = u0 + u1 + u2;
            const float cf = c[f];
            const float t3 = U * kThird;
            r[F[f][0]] = fmaf(-cf, fmaf(kFiveThirds, u0, t3), r[F[f][0]]);
            r[F[f][1]] = fmaf(-cf, fmaf(kFiveThirds, u1, t3), r[F[f][1]]);
            r[F[f][2]] = fmaf(-cf, fmaf(kFiveThirds, u2, t3), r[F[f][2]]);
            r[3 - f] = fmaf(cf * kFourThirds, U, r[3 - f]);
        }
    }
    const float4 A = T->a, B = T->b, S0 = T->s0;
    const float id = T->s1.x;
    const float v0 = (r[0] + r[1]) + (r[2] + r[3]);
    const float v1 = fmaf(B.x, r[0], fmaf(B.y, r[1], fmaf(B.z, r[2], B.w * r[3])));
    const float z0 = fmaf(S0.y, v0, -4.0f * v1) * S0.w;
    const float z1 = fmaf(S0.x, v1, -S0.z * v0) * S0.w;
    const float4 v = make_float4((r[0] - fmaf(A.x, z0, z1)) * id, (r[1] - fmaf(A.y, z0, z1)) * id,
                                 (r[2] - fmaf(A.z, z0, z1)) * id, (r[3] - fmaf(A.w, z0, z1)) * id);
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
__global__ void __launch_bounds__(1024) sweep_levels_kernel(SweepArgs a) {
    __shared__ float s_sigt[256];
    extern __shared__ float4 s_gtab_dyn[];
    load_sigt(a, s_sigt);
    const float4* s_gtab = load_gtab(a, s_gtab_dyn, s_sigt);
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
                        if (has[u]) assemble<false>(a, base, dir[d], item[u], s_sigt, up[u],
                                                    make_float4(0.f, 0.f, 0.f, 0.f), s_gtab);
#pragma unroll
                    for (int u = 0; u < ILP; ++u)
                        if (has[u]) finish<false>(base, item[u], up[u]);
                }
            }
            __syncthreads();
        }
    }
}

// Level-synchronous schedule with the next level's first item and source prefetched before the CTA
// barrier (they do not depend on the current level), so after the barrier only the geometry and
// the upstream values are waited for.  MINB = 2 asks for two 1024-thread CTAs per SM (32 registers).
template <int MINB>
__global__ void __launch_bounds__(1024, MINB) sweep_levels_pf_kernel(SweepArgs a) {
    __shared__ float s_sigt[256];
    extern __shared__ float4 s_gtab_dyn[];
    load_sigt(a, s_sigt);
    const float4* s_gtab = load_gtab(a, s_gtab_dyn, s_sigt);
    const int nt = blockDim.x;
    for (int i = blockIdx.x; i < a.NI; i += gridDim.x) {
        const int nl = __ldg(&a.nlev[i]);
        const int lb = __ldg(&a.lvl_base[i]);
        const float4 dir = __ldg(&a.dirs[i]);
        const int* it = a.items + (size_t)i * a.NE;
        float* base = a.psi + (size_t)i * (size_t)a.NENK;
        int s0 = __ldg(&a.lvl_start[lb]);
        int s1 = __ldg(&a.lvl_start[lb + 1]);
        // prefetched first update of this thread in the current level
        int pitem = (s0 + (int)threadIdx.x < s1) ? __ldcs(&it[s0 + threadIdx.x]) : 0;
        float4 pq = (s0 + (int)threadIdx.x < s1) ? *reinterpret_cast<const float4*>(base + 4 * (size_t)(pitem & 0xFFFFFF))
                                                 : make_float4(0.f, 0.f, 0.f, 0.f);
        for (int L = 0; L < nl; ++L) {
            const int es0 = s0 + threadIdx.x;
            const int cur_item = pitem;
            const float4 cur_q = pq;
            // next level bounds and prefetch (independent of this level's results)
            const int n0 = s1;
            const int n1 = (L + 1 < nl) ? __ldg(&a.lvl_start[lb + L + 2]) : s1;
            if (n0 + (int)threadIdx.x < n1) {
                pitem = __ldcs(&it[n0 + threadIdx.x]);
                pq = *reinterpret_cast<const float4*>(base + 4 * (size_t)(pitem & 0xFFFFFF));
            }
            if (es0 < s1) {
                Update up;
                assemble<false, true>(a, base, dir, cur_item, s_sigt, up, cur_q, s_gtab);
                finish<false>(base, cur_item, up);
            }
            for (int es = es0 + nt; es < s1; es += nt) {
                const int item = __ldcs(&it[es]);
                Update up;
                assemble<false>(a, base, dir, item, s_sigt, up, make_float4(0.f, 0.f, 0.f, 0.f), s_gtab);
                finish<false>(base, item, up);
            }
            s0 = n0;
            s1 = n1;
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Cluster schedule: blocks of kClusterSize consecutive elements (the 6 tets of a hex of a box mesh)
// swept as units.  The block graph of a direction is walked level by level with a CTA barrier
// between levels; a thread takes one block and updates its elements one after the other in their
// level order (an element's upstream neighbour inside the block was written by the same thread
// just before).  A block's sources and solutions are 96 contiguous bytes, read and written within a
// few hundred cycles, instead of six 16-byte accesses spread over several levels; and a direction
// has about a third as many block levels as element levels.  The element update is the level
// kernel's, so the results are bit-identical.
// ---------------------------------------------------------------------------------------------
template <int NT, int MINB, bool TAB, int PF>
__global__ void __launch_bounds__(NT, MINB) sweep_cluster_kernel(SweepArgs a) {
    __shared__ float s_sigt[256];
    extern __shared__ float4 s_gtab_dyn[];
    load_sigt(a, s_sigt);
    const float4* s_gtab = load_gtab(a, s_gtab_dyn, s_sigt);
    ElemTab* s_tab = reinterpret_cast<ElemTab*>(s_gtab_dyn + 3 * a.ngeom);   // TAB: [ngeom]
    const int nt = blockDim.x;
    for (int i = blockIdx.x; i < a.NI; i += gridDim.x) {
        const int nl = __ldg(&a.ncl[i]);
        const int* ls = a.cl_start + __ldg(&a.cl_base[i]);
        const float4 dir = __ldg(&a.dirs[i]);
        if (TAB) {
            __syncthreads();   // the previous direction's updates have read the table
            build_tab(s_gtab, s_sigt, a.ngeom, dir, s_tab);
            __syncthreads();
        }
        const int4* rec = a.crec + __ldg(&a.crec_base[i]);
        float* base = a.psi + (size_t)i * (size_t)a.NENK;
        int s1 = __ldg(&ls[0]);
        for (int L = 0; L < nl; ++L) {
            const int s0 = s1;
            s1 = __ldg(&ls[L + 1]);
            for (int cs = s0 + threadIdx.x; cs < s1; cs += nt) {
                const int4 r = __ldcs(rec + cs);
                const int e0 = r.x * kClusterSize;
                const int* mem = a.blk_elem ? a.blk_elem + e0 : nullptr;   // the block's members
                // slot fields, consumed 16 bits at a time from the low end
                unsigned long long pk = (unsigned long long)(unsigned)r.y | ((unsigned long long)(unsigned)r.z << 32);
                unsigned pw = (unsigned)r.w;
                if (PF && a.ngeom > 0) {
                    // The next element's record and source do not depend on the current update (the
                    // block's elements are distinct and only this thread writes them), so they are
                    // loaded one element ahead: the chain per element keeps only its upstream reads.
                    unsigned f = (unsigned)(pk & 0xFFFFu);
                    pk = (pk >> 16) | ((unsigned long long)(pw & 0xFFFFu) << 48);
                    pw >>= 16;
                    int e = mem ? __ldg(&mem[f & 7u]) : e0 + (int)(f & 7u);
                    int4 gn = __ldg(&a.rec[e]);
                    float4 q = ld4<false>(base + 4 * (size_t)e);
                    int prev_e = -1, prev2_e = -1;
                    float4 prev_v = make_float4(0.f, 0.f, 0.f, 0.f), prev2_v = prev_v;
#pragma unroll 1
                    for (int k = 0; k < kClusterSize; ++k) {
                        const unsigned fn = (unsigned)(pk & 0xFFFFu);
                        pk = (pk >> 16) | ((unsigned long long)(pw & 0xFFFFu) << 48);
                        pw >>= 16;
                        const bool more = k + 1 < kClusterSize && (fn & 7u) != 7u;
                        const int en = !more ? e : mem ? __ldg(&mem[fn & 7u]) : e0 + (int)(fn & 7u);
                        int4 gn_n = gn;
                        float4 q_n = q;
                        if (more) {
                            gn_n = __ldg(&a.rec[en]);
                            q_n = ld4<false>(base + 4 * (size_t)en);
                        }
                        const int item = e | (int)(((f >> 3) & 0xFu) << 24) | (int)(((f >> 7) & 0xFu) << 28);
                        if (TAB) {
                            update_tab_pre<false>(a, base, dir, item, gn, q, s_sigt, s_gtab, s_tab);
                        } else if (PF >= 2) {
                            Update up;
                            assemble_g<false, true, (PF >= 3 ? 2 : 1)>(base, dir, item, geom_from_rec(gn, s_gtab), s_sigt,
                                                                       up, q, prev_e, prev_v, prev2_e, prev2_v);
                            finish<false>(base, item, up);
                            if (PF >= 3) {
                                prev2_e = prev_e;
                                prev2_v = prev_v;
                            }
                            prev_e = e;
                            prev_v = make_float4(up.r[0], up.r[1], up.r[2], up.r[3]);
                        } else {
                            Update up;
                            assemble_g<false, true>(base, dir, item, geom_from_rec(gn, s_gtab), s_sigt, up, q);
                            finish<false>(base, item, up);
                        }
                        if (!more) break;
                        f = fn;
                        e = en;
                        gn = gn_n;
                        q = q_n;
                    }
                    continue;
                }
#pragma unroll 1
                for (int k = 0; k < kClusterSize; ++k) {
                    const unsigned f = (unsigned)(pk & 0xFFFFu);
                    pk = (pk >> 16) | ((unsigned long long)(pw & 0xFFFFu) << 48);
                    pw >>= 16;
                    if ((f & 7u) == 7u) break;
                    const int eo = mem ? __ldg(&mem[f & 7u]) : e0 + (int)(f & 7u);
                    const int item = eo | (int)(((f >> 3) & 0xFu) << 24) | (int)(((f >> 7) & 0xFu) << 28);
                    if (TAB) {
                        update_tab<false>(a, base, dir, item, s_sigt, s_gtab, s_tab);
                    } else {
                        Update up;
                        assemble<false>(a, base, dir, item, s_sigt, up, make_float4(0.f, 0.f, 0.f, 0.f), s_gtab);
                        finish<false>(base, item, up);
                    }
                }
            }
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Batched level schedule: one persistent launch over the directions of many independent problems
// (meshes, quadratures and cross sections differ).  A direction whose problem has a block schedule is
// walked block level by block level, as the cluster kernel does, with the problem's element types
// staged in shared memory.  CTAs claim work items in order from a global
// counter, so items sorted by decreasing cost give a longest-first list schedule; each item is a
// whole direction walked level by level with a CTA barrier between levels, exactly like the
// single-problem level kernel (same element update, bit-identical results).
// ---------------------------------------------------------------------------------------------
template <int NT>
__global__ void __launch_bounds__(NT, NT >= 1024 ? 1 : 2) sweep_batch_kernel(const BatchWork* __restrict__ work, int nwork, int* counter,
                                                        const int* __restrict__ active) {
    __shared__ float s_sigt[256];
    __shared__ float4 s_gt[3 * 256];   // the item's element types (face vectors), when it has a type table
    __shared__ int s_w;
    for (;;) {
        if (threadIdx.x == 0) s_w = atomicAdd(counter, 1);
        __syncthreads();
        const int w = s_w;
        if (w >= nwork) return;
        const BatchWork* W = work + w;
        const int prob = __ldg(&W->problem);
        if (active && __ldg(&active[prob]) == 0) {
            __syncthreads();
            continue;
        }
        const int Nm = __ldg(&W->Nm);
        const float* sg = W->sigt;
        const int ngeom = __ldg(&W->ngeom);
        const int4* crec = W->crec;
        // cross sections by material, or by element type when the problem has a type table
        for (int m = threadIdx.x; m < 256; m += NT) {
            float v = 0.f;
            if (ngeom > 0) v = (m < ngeom) ? __ldg(&sg[__ldg(&W->tmat[m])]) : 0.f;
            else v = (m < Nm) ? __ldg(&sg[m]) : 0.f;
            s_sigt[m] = v;
        }
        for (int k = threadIdx.x; k < 3 * ngeom; k += NT) s_gt[k] = __ldg(&W->gtab[k]);
        const int nl = __ldg(&W->nlev);
        const int* ls = W->lvl_start;
        const int* it = W->items;
        const float4* geom = W->geom;
        float* base = W->psi;
        const float4 dir = __ldg(&W->dir);
        __syncthreads();
        if (crec) {
            // block schedule, as sweep_cluster_kernel
            const int ncl = __ldg(&W->ncl);
            const int* cls = W->cl_start;
            const int4* rec = W->rec;
            for (int L = 0; L < ncl; ++L) {
                const int s0 = __ldg(&cls[L]), s1 = __ldg(&cls[L + 1]);
                for (int cs = s0 + threadIdx.x; cs < s1; cs += NT) {
                    const int4 r = __ldcs(crec + cs);
                    const int e0 = r.x * kClusterSize;
                    const int* mem = W->blk_elem ? W->blk_elem + e0 : nullptr;
                    unsigned long long pk = (unsigned long long)(unsigned)r.y | ((unsigned long long)(unsigned)r.z << 32);
                    unsigned pw = (unsigned)r.w;
                    if (ngeom > 0) {
                        // the cluster kernel's walk: next element's record and source loaded one element
                        // ahead, the two previous solutions kept in registers for upstream reads in the block
                        unsigned f = (unsigned)(pk & 0xFFFFu);
                        pk = (pk >> 16) | ((unsigned long long)(pw & 0xFFFFu) << 48);
                        pw >>= 16;
                        int e = mem ? __ldg(&mem[f & 7u]) : e0 + (int)(f & 7u);
                        int4 gn = __ldg(&rec[e]);
                        float4 q = ld4<false>(base + 4 * (size_t)e);
                        int prev_e = -1, prev2_e = -1;
                        float4 prev_v = make_float4(0.f, 0.f, 0.f, 0.f), prev2_v = prev_v;
#pragma unroll 1
                        for (int k = 0; k < kClusterSize; ++k) {
                            const unsigned fn = (unsigned)(pk & 0xFFFFu);
                            pk = (pk >> 16) | ((unsigned long long)(pw & 0xFFFFu) << 48);
                            pw >>= 16;
                            const bool more = k + 1 < kClusterSize && (fn & 7u) != 7u;
                            const int en = !more ? e : mem ? __ldg(&mem[fn & 7u]) : e0 + (int)(fn & 7u);
                            int4 gn_n = gn;
                            float4 q_n = q;
                            if (more) {
                                gn_n = __ldg(&rec[en]);
                                q_n = ld4<false>(base + 4 * (size_t)en);
                            }
                            const int item = e | (int)(((f >> 3) & 0xFu) << 24) | (int)(((f >> 7) & 0xFu) << 28);
                            Update up;
                            assemble_g<false, true, 2>(base, dir, item, geom_from_rec(gn, s_gt), s_sigt, up, q, prev_e,
                                                       prev_v, prev2_e, prev2_v);
                            finish<false>(base, item, up);
                            prev2_e = prev_e;
                            prev2_v = prev_v;
                            prev_e = e;
                            prev_v = make_float4(up.r[0], up.r[1], up.r[2], up.r[3]);
                            if (!more) break;
                            f = fn;
                            e = en;
                            gn = gn_n;
                            q = q_n;
                        }
                        continue;
                    }
#pragma unroll 1
                    for (int k = 0; k < kClusterSize; ++k) {
                        const unsigned f = (unsigned)(pk & 0xFFFFu);
                        pk = (pk >> 16) | ((unsigned long long)(pw & 0xFFFFu) << 48);
                        pw >>= 16;
                        if ((f & 7u) == 7u) break;
                        const int e = mem ? __ldg(&mem[f & 7u]) : e0 + (int)(f & 7u);
                        const int item = e | (int)(((f >> 3) & 0xFu) << 24) | (int)(((f >> 7) & 0xFu) << 28);
                        const Geom g = load_geom(geom, e);
                        Update up;
                        assemble_g<false>(base, dir, item, g, s_sigt, up, make_float4(0.f, 0.f, 0.f, 0.f));
                        finish<false>(base, item, up);
                    }
                }
                __syncthreads();
            }
            continue;
        }
        for (int L = 0; L < nl; ++L) {
            const int s0 = __ldg(&ls[L]), s1 = __ldg(&ls[L + 1]);
            for (int es = s0 + threadIdx.x; es < s1; es += NT) {
                const int item = __ldcs(&it[es]);
                const Geom g = load_geom(geom, item & 0xFFFFFF);
                Update up;
                assemble_g<false>(base, dir, item, g, s_sigt, up, make_float4(0.f, 0.f, 0.f, 0.f));
                finish<false>(base, item, up);
            }
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Element-flag schedule: one CTA per direction, no barriers between levels.  Warps claim 32-element
// chunks of the direction's padded sweep order (levels padded to multiples of 32, so a chunk's
// elements are mutually independent) from a shared counter, prefetch the next chunk's items,
// geometry and source, and wait -- bounded -- only for the done bits of their own upstream
// neighbours (one bit per element in shared memory).  Claims are made in sweep order and every
// dependency lies earlier in that order, so the earliest unfinished chunk can always proceed.
// ---------------------------------------------------------------------------------------------
template <int NT>
__global__ void __launch_bounds__(NT, NT >= 1024 ? 1 : 2) sweep_flags_kernel(SweepArgs a) {
    extern __shared__ uint32_t s_done[];                      // one bit per element of the mesh
    __shared__ float s_sigt[256];
    __shared__ int s_next;
    __shared__ int s_abort;
    __shared__ int s_ndone, s_nexit;
    load_sigt(a, s_sigt);
    const int lane = threadIdx.x & 31;
    const int nwords = (a.NE + 31) >> 5;
    volatile uint32_t* vdone = s_done;
    for (int i = blockIdx.x; i < a.NI; i += gridDim.x) {
        for (int w = threadIdx.x; w < nwords; w += NT) s_done[w] = 0u;
        if (threadIdx.x == 0) { s_next = 0; s_abort = 0; s_ndone = 0; s_nexit = 0; }
        __syncthreads();
        const long long pb = __ldg(&a.pbase[i]);
        const int len = (int)(__ldg(&a.pbase[i + 1]) - pb);
        const int* pit = a.pitems + pb;
        const float4 dir = __ldg(&a.dirs[i]);
        float* base = a.psi + (size_t)i * (size_t)a.NENK;
        int c = 0;
        if (lane == 0) c = atomicAdd(&s_next, 32);
        c = __shfl_sync(0xffffffffu, c, 0);
        int item = -1;
        Geom G;
        float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
        if (c < len) {
            item = __ldcs(&pit[c + lane]);
            if (item != kPad) { G = load_geom(a.geom, item & 0xFFFFFF); q = *reinterpret_cast<const float4*>(base + 4 * (size_t)(item & 0xFFFFFF)); }
        }
        while (c < len) {
            int cn = 0;
            if (lane == 0) cn = atomicAdd(&s_next, 32);
            cn = __shfl_sync(0xffffffffu, cn, 0);
            int nitem = -1;
            Geom NG;
            float4 nq = make_float4(0.f, 0.f, 0.f, 0.f);
            if (cn < len) {
                nitem = __ldcs(&pit[cn + lane]);
                if (nitem != kPad) { NG = load_geom(a.geom, nitem & 0xFFFFFF); nq = *reinterpret_cast<const float4*>(base + 4 * (size_t)(nitem & 0xFFFFFF)); }
            }
            bool ok = true;
            if (item != kPad) {
                // wait for the upstream neighbours of this element
                const int upm = (item >> 24) & 0xF;
                const unsigned nw[4] = {(unsigned)G.gn.x, (unsigned)G.gn.y, (unsigned)G.gn.z, (unsigned)G.gn.w};
                long long spins = 0;
                int waited = -1;
#pragma unroll
                for (int f = 0; f < 4; ++f) {
                    if (!((upm >> f) & 1)) continue;
                    const int ep = (int)(nw[f] & 0xFFFFFFu);
                    const uint32_t bit = 1u << (ep & 31);
                    while (!(vdone[ep >> 5] & bit)) {
                        if (++spins > a.spin_limit || *((volatile int*)&s_abort)) { ok = false; waited = ep; break; }
                        __nanosleep(32);
                    }
                    if (!ok) break;
                }
                if (ok) {
                    __threadfence_block();
                    Update u;
                    assemble_g<false, true>(base, dir, item, G, s_sigt, u, q);
                    finish<false>(base, item, u);
                    __threadfence_block();
                    const int e = item & 0xFFFFFF;
                    atomicOr(&s_done[e >> 5], 1u << (e & 31));
                    atomicAdd(&s_ndone, 1);
                } else if (atomicExch(&s_abort, 1) == 0) {
                    if (atomicExch(&a.status->abort, 1) == 0) {
                        a.status->err = LB_ERR_TIMEOUT;
                        a.status->err_chunk = i;
                        a.status->err_elem = item & 0xFFFFFF;
                        a.status->err_dep = waited;
                        a.status->err_pos = c;
                        a.status->err_bit = waited >= 0 ? (int)((vdone[waited >> 5] >> (waited & 31)) & 1u) : -1;
                        a.status->dbg_next = *((volatile int*)&s_next);
                        a.status->dbg_done = *((volatile int*)&s_ndone);
                        a.status->dbg_exited = *((volatile int*)&s_nexit);
                        a.status->dbg_len = len;
                    }
                }
            }
            if (__any_sync(0xffffffffu, !ok) || *((volatile int*)&s_abort)) break;
            c = cn;
            item = nitem;
            G = NG;
            q = nq;
        }
        if (lane == 0) atomicAdd(&s_nexit, 1);
        __syncthreads();
        if (*((volatile int*)&s_abort)) return;
    }
}

// ---------------------------------------------------------------------------------------------
// Grouped level schedule: directions whose schedules are bit-identical (same order and same face
// masks for every element) are walked together.  Each element's item and geometry are loaded once
// for the group, the group's source and upstream values are all requested before any of its
// updates is computed, so the memory latency of one element is paid once for G directions.
// groups: per CTA work item {representative direction, count, d0 .. d5}.
// ---------------------------------------------------------------------------------------------
template <int G>
__device__ __forceinline__ void group_update(const SweepArgs& a, float* const* base, const float4* dir, int n, int item,
                                             const float* s_sigt) {
    constexpr int F[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
    const int e = item & 0xFFFFFF;
    const int upm = (item >> 24) & 0xF;
    const int outm = (item >> 28) & 0xF;
    const Geom g = load_geom(a.geom, e);
    const unsigned nw[4] = {(unsigned)g.gn.x, (unsigned)g.gn.y, (unsigned)g.gn.z, (unsigned)g.gn.w};
    // request every direction's source and upstream values first
    float4 q[G], up[G][4];
#pragma unroll
    for (int j = 0; j < G; ++j) {
        if (j >= n) break;
        q[j] = *reinterpret_cast<const float4*>(base[j] + 4 * (size_t)e);
#pragma unroll
        for (int f = 0; f < 4; ++f)
            if ((upm >> f) & 1) up[j][f] = *reinterpret_cast<const float4*>(base[j] + 4 * (size_t)(nw[f] & 0xFFFFFFu));
    }
    const int matid = (int)((nw[0] >> 30) | ((nw[1] >> 30) << 2) | ((nw[2] >> 30) << 4) | ((nw[3] >> 30) << 6));
    const float sig = s_sigt[matid];
#pragma unroll
    for (int j = 0; j < G; ++j) {
        if (j >= n) break;
        const float4 d = dir[j];
        float c[4];
        c[0] = fmaf(d.x, g.gx.x, fmaf(d.y, g.gy.x, d.z * g.gz.x));
        c[1] = fmaf(d.x, g.gx.y, fmaf(d.y, g.gy.y, d.z * g.gz.y));
        c[2] = fmaf(d.x, g.gx.z, fmaf(d.y, g.gy.z, d.z * g.gz.z));
        c[3] = fmaf(d.x, g.gx.w, fmaf(d.y, g.gy.w, d.z * g.gz.w));
        Update u;
        u.r[0] = q[j].x; u.r[1] = q[j].y; u.r[2] = q[j].z; u.r[3] = q[j].w;
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            if ((upm >> f) & 1) {
                const unsigned wd = nw[f];
                const float u0 = pick(up[j][f], (wd >> 24) & 3);
                const float u1 = pick(up[j][f], (wd >> 26) & 3);
                const float u2 = pick(up[j][f], (wd >> 28) & 3);
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
        solve_rank2(u);
        *reinterpret_cast<float4*>(base[j] + 4 * (size_t)e) = make_float4(u.r[0], u.r[1], u.r[2], u.r[3]);
    }
}

template <int G, int NT>
__global__ void __launch_bounds__(NT, 1) sweep_group_kernel(SweepArgs a, const int* __restrict__ groups, int ngroups) {
    __shared__ float s_sigt[256];
    load_sigt(a, s_sigt);
    for (int gi = blockIdx.x; gi < ngroups; gi += gridDim.x) {
        const int* gr = groups + (size_t)gi * 8;
        const int rep = __ldg(&gr[0]);
        const int n = __ldg(&gr[1]);
        float* base[G];
        float4 dir[G];
#pragma unroll
        for (int j = 0; j < G; ++j) {
            const int i = (j < n) ? __ldg(&gr[2 + j]) : rep;
            base[j] = a.psi + (size_t)i * (size_t)a.NENK;
            dir[j] = __ldg(&a.dirs[i]);
        }
        const int nl = __ldg(&a.nlev[rep]);
        const int lb = __ldg(&a.lvl_base[rep]);
        const int* it = a.items + (size_t)rep * a.NE;
        for (int L = 0; L < nl; ++L) {
            const int s0 = __ldg(&a.lvl_start[lb + L]);
            const int s1 = __ldg(&a.lvl_start[lb + L + 1]);
            for (int es = s0 + threadIdx.x; es < s1; es += NT) group_update<G>(a, base, dir, n, __ldcs(&it[es]), s_sigt);
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
    int kind;      // 0 levels, 1 dataflow, 2 levels with next-level prefetch, 3 element flags, 4 grouped levels,
                   // 5 blocks of elements (cluster records), 6 the same with per-type element tables
    int threads;
    int dpc;       // directions per CTA (kind 0); minimum CTAs per SM (kinds 2, 5)
    int ilp;       // updates in flight per thread (kind 0); kinds 5, 6: 2 = next element's record and source
                   // prefetched, 3 = the same and the previous element's solution kept in registers, 4 = the
                   // same with the two previous elements' solutions
};

const Config kConfigs[] = {
    {4, 1024, 2, 1}, {4, 512, 2, 1}, {4, 512, 3, 1}, {4, 1024, 3, 1}, {4, 512, 6, 1},
    {0, 1024, 1, 1}, {0, 512, 1, 1}, {2, 1024, 1, 1}, {3, 512, 0, 1}, {1, 256, 0, 0},
    {4, 768, 2, 1}, {0, 1024, 1, 2}, {0, 1024, 1, 3}, {0, 768, 1, 3}, {5, 1024, 1, 1}, {5, 512, 2, 1}, {5, 768, 2, 1}, {5, 1024, 2, 1},
    {6, 512, 2, 1}, {6, 768, 2, 1}, {5, 512, 2, 2}, {6, 512, 2, 2}, {5, 512, 2, 3}, {5, 512, 2, 4},
};
constexpr int kNumConfigs = sizeof(kConfigs) / sizeof(kConfigs[0]);
constexpr int kFinalists = 3;   // candidates timed a second time before one is kept

template <int DPC, int ILP>
cudaError_t launch_levels(const SweepArgs& a, int threads, int sm_count, cudaStream_t s) {
    const size_t smem = sizeof(float4) * 3 * (size_t)a.ngeom;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sweep_levels_kernel<DPC, ILP>, threads, smem);
    if (per_sm < 1) per_sm = 1;
    int ctas = (a.NI + DPC - 1) / DPC;
    int grid = std::min(ctas, sm_count * per_sm);
    sweep_levels_kernel<DPC, ILP><<<grid, threads, smem, s>>>(a);
    return cudaGetLastError();
}

template <int G, int NT>
cudaError_t launch_group(const SweepArgs& a, const int* groups, int ngroups, int sm_count, cudaStream_t s) {
    static PerDevice per_sm_cache;
    const int per_sm = per_sm_cache.get([&] {
        int n = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sweep_group_kernel<G, NT>, NT, 0);
        return n < 1 ? 1 : n;
    });
    int grid = std::min(ngroups, sm_count * per_sm);
    sweep_group_kernel<G, NT><<<grid, NT, 0, s>>>(a, groups, ngroups);
    return cudaGetLastError();
}

// per-CTA groups of at most gmax directions with identical schedules
int build_groups(Handle* h, int gmax) {
    if (h->groups_gmax == gmax && h->d_groups) return LB_OK;
    std::vector<int> gr;
    int ng = 0;
    for (size_t c = 0; c + 1 < h->class_start.size(); ++c) {
        const int a0 = h->class_start[c], a1 = h->class_start[c + 1];
        for (int s = a0; s < a1; s += gmax) {
            const int n = std::min(gmax, a1 - s);
            int rec[8] = {h->class_members[a0], n, 0, 0, 0, 0, 0, 0};
            for (int j = 0; j < n; ++j) rec[2 + j] = h->class_members[s + j];
            gr.insert(gr.end(), rec, rec + 8);
            ++ng;
        }
    }
    if (h->d_groups) { cudaFree(h->d_groups); h->d_groups = nullptr; }
    cudaError_t e = cudaMalloc(&h->d_groups, sizeof(int) * gr.size());
    if (e == cudaSuccess) e = cudaMemcpy(h->d_groups, gr.data(), sizeof(int) * gr.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(h, e, "sweep groups");
    h->groups_gmax = gmax;
    h->ngroups = ng;
    const char* verbose = std::getenv("LB_SWEEP_VERBOSE");
    if (verbose && *verbose == '1')
        std::fprintf(stderr, "sweep: %d directions in %zu schedule classes -> %d groups of <= %d\n", h->NI,
                     h->class_start.size() - 1, ng, gmax);
    return LB_OK;
}

template <int NT>
cudaError_t launch_flags(const SweepArgs& a, int sm_count, cudaStream_t s) {
    const size_t smem = sizeof(uint32_t) * (size_t)((a.NE + 31) / 32);
    if (smem > 200 * 1024) return cudaErrorInvalidConfiguration;
    static PerDevice attr;
    attr.get([&] {
        allow_max_dynamic_smem(sweep_flags_kernel<NT>);
        return 1;
    });
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sweep_flags_kernel<NT>, NT, smem);
    if (per_sm < 1) per_sm = 1;
    int grid = std::min(a.NI, sm_count * per_sm);
    sweep_flags_kernel<NT><<<grid, NT, smem, s>>>(a);
    return cudaGetLastError();
}

template <int NT, int MINB, bool TAB, int PF = 0>
cudaError_t launch_cluster(const SweepArgs& a, int sm_count, cudaStream_t s) {
    const size_t smem = (sizeof(float4) * 3 + (TAB ? sizeof(ElemTab) : 0)) * (size_t)a.ngeom;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sweep_cluster_kernel<NT, MINB, TAB, PF>, NT, smem);
    if (per_sm < 1) per_sm = 1;
    int grid = std::min(a.NI, sm_count * per_sm);
    sweep_cluster_kernel<NT, MINB, TAB, PF><<<grid, NT, smem, s>>>(a);
    return cudaGetLastError();
}

template <int MINB>
cudaError_t launch_levels_pf(const SweepArgs& a, int threads, int sm_count, cudaStream_t s) {
    const size_t smem = sizeof(float4) * 3 * (size_t)a.ngeom;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sweep_levels_pf_kernel<MINB>, threads, smem);
    if (per_sm < 1) per_sm = 1;
    int grid = std::min(a.NI, sm_count * per_sm);
    sweep_levels_pf_kernel<MINB><<<grid, threads, smem, s>>>(a);
    return cudaGetLastError();
}

}  // namespace

int launch_sweep_batch(cudaStream_t st, const BatchWork* work, int nwork, int* counter, const int* active, int threads,
                       int sm_count) {
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(int), st);
    if (e != cudaSuccess) return LB_ERR_CUDA;
    if (threads == 512) {
        static PerDevice per_sm_cache;
        const int per_sm = per_sm_cache.get([&] {
            int n = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sweep_batch_kernel<512>, 512, 0);
            return n < 1 ? 1 : n;
        });
        sweep_batch_kernel<512><<<std::min(nwork, sm_count * per_sm), 512, 0, st>>>(work, nwork, counter, active);
    } else {
        static PerDevice per_sm_cache;
        const int per_sm = per_sm_cache.get([&] {
            int n = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sweep_batch_kernel<1024>, 1024, 0);
            return n < 1 ? 1 : n;
        });
        sweep_batch_kernel<1024><<<std::min(nwork, sm_count * per_sm), 1024, 0, st>>>(work, nwork, counter, active);
    }
    return cudaGetLastError() == cudaSuccess ? LB_OK : LB_ERR_CUDA;
}

int launch_sweep(Handle* h, float* psi) {
    SweepArgs a{};
    a.items = h->d_items;
    a.pitems = h->d_pitems;
    a.pbase = h->d_pbase;
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
    a.rec = h->d_rec;
    a.gtab = h->d_gtab;
    a.tmat = h->d_tmat;
    a.ngeom = h->ngeom;
    a.crec = h->d_crec;
    a.crec_base = h->d_crec_base;
    a.blk_elem = h->d_blk_elem;
    a.cl_start = h->d_cl_start;
    a.cl_base = h->d_cl_base;
    a.ncl = h->d_ncl;
    a.nclusters = h->nclusters;

    if (h->sweep_cfg_forced < 0) {
        const char* env = std::getenv("LB_SWEEP_CONFIG");
        h->sweep_cfg_forced = (env && *env) ? std::atoi(env) : kNumConfigs;
        if (h->sweep_cfg_forced < 0) h->sweep_cfg_forced = kNumConfigs;
    }
    int cfg_idx;
    bool tuning = false;
    if (h->sweep_cfg_forced < kNumConfigs) cfg_idx = h->sweep_cfg_forced;
    else if (h->sweep_cfg >= 0) cfg_idx = h->sweep_cfg;
    else {
        // a first pass times every candidate once; a second pass times the kFinalists fastest once more
        cfg_idx = h->sweep_trial < kNumConfigs ? h->sweep_trial : h->sweep_finalists[h->sweep_trial - kNumConfigs];
        tuning = true;
    }
    if (tuning && h->sweep_trial == 0) {
        // load every candidate's module before timing, so the first trial does not pay for it
        cudaFuncAttributes fa;
        cudaFuncGetAttributes(&fa, sweep_group_kernel<2, 1024>);
        cudaFuncGetAttributes(&fa, sweep_group_kernel<2, 512>);
        cudaFuncGetAttributes(&fa, sweep_group_kernel<3, 1024>);
        cudaFuncGetAttributes(&fa, sweep_group_kernel<3, 512>);
        cudaFuncGetAttributes(&fa, sweep_group_kernel<6, 512>);
        cudaFuncGetAttributes(&fa, sweep_flags_kernel<256>);
        cudaFuncGetAttributes(&fa, sweep_flags_kernel<512>);
        cudaFuncGetAttributes(&fa, sweep_flags_kernel<1024>);
        cudaFuncGetAttributes(&fa, sweep_levels_pf_kernel<1>);
        cudaFuncGetAttributes(&fa, sweep_levels_pf_kernel<2>);
        cudaFuncGetAttributes(&fa, sweep_levels_kernel<1, 1>);
        cudaFuncGetAttributes(&fa, sweep_levels_kernel<1, 2>);
        cudaFuncGetAttributes(&fa, sweep_levels_kernel<1, 3>);
        cudaFuncGetAttributes(&fa, sweep_levels_kernel<2, 1>);
        cudaFuncGetAttributes(&fa, sweep_levels_kernel<2, 2>);
        cudaFuncGetAttributes(&fa, sweep_dataflow_kernel);
        cudaFuncGetAttributes(&fa, sweep_group_kernel<2, 768>);
        cudaFuncGetAttributes(&fa, sweep_cluster_kernel<1024, 1, false, 0>);
        cudaFuncGetAttributes(&fa, sweep_cluster_kernel<1024, 2, false, 0>);
        cudaFuncGetAttributes(&fa, sweep_cluster_kernel<768, 2, false, 0>);
        cudaFuncGetAttributes(&fa, sweep_cluster_kernel<512, 2, false, 0>);
        cudaFuncGetAttributes(&fa, sweep_cluster_kernel<512, 2, true, 0>);
        cudaFuncGetAttributes(&fa, sweep_cluster_kernel<768, 2, true, 0>);
        cudaFuncGetAttributes(&fa, sweep_cluster_kernel<512, 2, false, 1>);
        cudaFuncGetAttributes(&fa, sweep_cluster_kernel<512, 2, true, 1>);
        cudaFuncGetAttributes(&fa, sweep_cluster_kernel<512, 2, false, 2>);
        cudaFuncGetAttributes(&fa, sweep_cluster_kernel<512, 2, false, 3>);
    }
    Config cfg = kConfigs[cfg_idx];
    // the autotuner skips the block schedule where it has more barrier levels than the element schedule
    // (unstructured meshes, whose blocks are split on cycles): it cannot win there; a forced
    // configuration still runs it
    if ((cfg.kind == 5 || cfg.kind == 6) && h->sweep_cfg_forced >= kNumConfigs &&
        h->cluster_levels_total > (long long)h->total_levels)
        cfg = Config{0, 1024, 1, 2};
    // the element-flag schedule keeps one bit per element in shared memory
    if (cfg.kind == 3 && (size_t)((h->NE + 31) / 32) * 4 > 200 * 1024) cfg = Config{0, 1024, 1, 1};
    // the cluster schedule needs block records (built when every direction's block graph is acyclic)
    if (cfg.kind == 5 && h->nclusters <= 0) cfg = Config{0, 1024, 1, 2};
    // per-type element tables need the type table as well
    if (cfg.kind == 6 && (h->nclusters <= 0 || h->ngeom <= 0))
        cfg = h->nclusters > 0 ? Config{5, 512, 2, 1} : Config{0, 1024, 1, 2};

    cudaError_t e = cudaSuccess;
    if (cfg.kind == 1) {
        e = cudaMemsetAsync(h->d_done, 0, sizeof(int) * (size_t)h->total_levels, h->stream);
        if (e != cudaSuccess) return cuda_fail(h, e, "sweep: reset counters");
    }
    if (cfg.kind == 1 || cfg.kind == 3) {
        e = cudaMemsetAsync(h->d_status, 0, sizeof(SweepStatus), h->stream);
        if (e != cudaSuccess) return cuda_fail(h, e, "sweep: reset status");
    }
    if (cfg.kind == 4) {
        int rc = build_groups(h, cfg.dpc);
        if (rc) return rc;
    }
    Timer t;
    timer_begin(h, LB_T_SWEEP, t);
    if (cfg.kind == 4) {
        if (cfg.dpc == 2) e = cfg.threads == 1024 ? launch_group<2, 1024>(a, h->d_groups, h->ngroups, h->sm_count, h->stream)
                            : cfg.threads == 768 ? launch_group<2, 768>(a, h->d_groups, h->ngroups, h->sm_count, h->stream)
                                                 : launch_group<2, 512>(a, h->d_groups, h->ngroups, h->sm_count, h->stream);
        else if (cfg.dpc == 3) e = cfg.threads == 1024 ? launch_group<3, 1024>(a, h->d_groups, h->ngroups, h->sm_count, h->stream)
                                                       : launch_group<3, 512>(a, h->d_groups, h->ngroups, h->sm_count, h->stream);
        else e = launch_group<6, 512>(a, h->d_groups, h->ngroups, h->sm_count, h->stream);
    } else if (cfg.kind == 3) {
        e = (cfg.threads == 256) ? launch_flags<256>(a, h->sm_count, h->stream)
          : (cfg.threads == 1024) ? launch_flags<1024>(a, h->sm_count, h->stream)
                                  : launch_flags<512>(a, h->sm_count, h->stream);
    } else if ((cfg.kind == 5 || cfg.kind == 6) && cfg.ilp >= 2) {
        e = cfg.kind == 6   ? launch_cluster<512, 2, true, 1>(a, h->sm_count, h->stream)
            : cfg.ilp == 4 ? launch_cluster<512, 2, false, 3>(a, h->sm_count, h->stream)
            : cfg.ilp == 3 ? launch_cluster<512, 2, false, 2>(a, h->sm_count, h->stream)
                           : launch_cluster<512, 2, false, 1>(a, h->sm_count, h->stream);
    } else if (cfg.kind == 5) {
        if (cfg.threads == 1024) e = cfg.dpc == 2 ? launch_cluster<1024, 2, false>(a, h->sm_count, h->stream)
                                                  : launch_cluster<1024, 1, false>(a, h->sm_count, h->stream);
        else if (cfg.threads == 768) e = launch_cluster<768, 2, false>(a, h->sm_count, h->stream);
        else e = launch_cluster<512, 2, false>(a, h->sm_count, h->stream);
    } else if (cfg.kind == 6) {
        e = cfg.threads == 768 ? launch_cluster<768, 2, true>(a, h->sm_count, h->stream)
                               : launch_cluster<512, 2, true>(a, h->sm_count, h->stream);
    } else if (cfg.kind == 2) {
        e = (cfg.dpc == 2) ? launch_levels_pf<2>(a, cfg.threads, h->sm_count, h->stream)
                           : launch_levels_pf<1>(a, cfg.threads, h->sm_count, h->stream);
    } else if (cfg.kind == 1) {
        static PerDevice df_per_sm_cache;
        const int df_per_sm = df_per_sm_cache.get([&] {
            int n = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sweep_dataflow_kernel, 256, 0);
            return n < 1 ? 1 : n;
        });
        sweep_dataflow_kernel<<<h->sm_count * df_per_sm, 256, 0, h->stream>>>(a);
        e = cudaGetLastError();
    } else if (cfg.dpc == 1 && cfg.ilp == 1) e = launch_levels<1, 1>(a, cfg.threads, h->sm_count, h->stream);
    else if (cfg.dpc == 1 && cfg.ilp == 2) e = launch_levels<1, 2>(a, cfg.threads, h->sm_count, h->stream);
    else if (cfg.dpc == 1 && cfg.ilp == 3) e = launch_levels<1, 3>(a, cfg.threads, h->sm_count, h->stream);
    else if (cfg.dpc == 2 && cfg.ilp == 1) e = launch_levels<2, 1>(a, cfg.threads, h->sm_count, h->stream);
    else e = launch_levels<2, 2>(a, cfg.threads, h->sm_count, h->stream);
    timer_end(h, t);
    if (e != cudaSuccess) return cuda_fail(h, e, "sweep kernel launch");
    if (cfg.kind == 1 || cfg.kind == 3) {
        SweepStatus st;
        e = cudaMemcpyAsync(&st, h->d_status, sizeof(st), cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) return cuda_fail(h, e, "sweep kernel");
        if (st.err) {
            char buf[256];
            if (cfg.kind == 3)
                std::snprintf(buf, sizeof buf, "sweep: dependency wait timed out in direction %d: element %d waited for "
                              "element %d (bit %d), chunk at %d; claimed %d of %d, completed %d, warps exited %d",
                              st.err_chunk, st.err_elem, st.err_dep, st.err_bit, st.err_pos, st.dbg_next, st.dbg_len,
                              st.dbg_done, st.dbg_exited);
            else
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
        ++h->sweep_trial;
        if (h->sweep_trial == kNumConfigs) {
            std::vector<int> order(kNumConfigs);
            for (int c = 0; c < kNumConfigs; ++c) order[c] = c;
            std::stable_sort(order.begin(), order.end(),
                             [&](int x, int y) { return h->sweep_trial_ms[x] < h->sweep_trial_ms[y]; });
            h->sweep_finalists.assign(order.begin(), order.begin() + std::min(kFinalists, kNumConfigs));
        }
        const int nfin = (int)h->sweep_finalists.size();
        if (h->sweep_trial == kNumConfigs + nfin) {
            // the finalist with the smallest sum of its two times (one noisy sweep decides nothing)
            int best = -1;
            float best_ms = 0.f;
            for (int q = 0; q < nfin; ++q) {
                const int c = h->sweep_finalists[q];
                const float tot = h->sweep_trial_ms[c] + h->sweep_trial_ms[kNumConfigs + q];
                if (best < 0 || tot < best_ms) { best = c; best_ms = tot; }
            }
            h->sweep_cfg = best;
            const char* verbose = std::getenv("LB_SWEEP_VERBOSE");
            if (verbose && *verbose == '1')
                for (int c = 0; c < kNumConfigs; ++c) {
                    float again = -1.f;
                    for (int q = 0; q < nfin; ++q)
                        if (h->sweep_finalists[q] == c) again = h->sweep_trial_ms[kNumConfigs + q];
                    std::fprintf(stderr, "sweep config %d (kind %d threads %d dpc %d ilp %d): %.3f ms", c, kConfigs[c].kind,
                                 kConfigs[c].threads, kConfigs[c].dpc, kConfigs[c].ilp, h->sweep_trial_ms[c]);
                    if (again >= 0.f) std::fprintf(stderr, ", again %.3f ms", again);
                    std::fprintf(stderr, "%s\n", c == best ? "  <- chosen" : "");
                }
        }
    }
    return LB_OK;
}

int sweep_config(Handle* h, int* kind, int* threads, int* dpc, int* ilp) {
    int c = h->sweep_cfg_forced >= 0 && h->sweep_cfg_forced < kNumConfigs ? h->sweep_cfg_forced : h->sweep_cfg;
    if (c < 0) return -1;
    Config cfg = kConfigs[c];
    if ((cfg.kind == 5 || cfg.kind == 6) && h->sweep_cfg_forced >= kNumConfigs &&
        h->cluster_levels_total > (long long)h->total_levels)
        cfg = Config{0, 1024, 1, 2};   // what the launcher runs instead
    if (cfg.kind == 5 && h->nclusters <= 0) cfg = Config{0, 1024, 1, 2};   // what the launcher runs instead
    if (cfg.kind == 6 && (h->nclusters <= 0 || h->ngeom <= 0))
        cfg = h->nclusters > 0 ? Config{5, 512, 2, 1} : Config{0, 1024, 1, 2};
    *kind = cfg.kind; *threads = cfg.threads; *dpc = cfg.dpc; *ilp = cfg.ilp;
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
//  It always runs the dataflow schedule (sweep_dataflow_kernel), whose only scratch is these
//  counters, not the schedule the autotuner picks for lb_transport_inv, so its timing differs.
//  The call is synchronous on the handle's stream (it reads the status block back), so it cannot
//  be stream-captured, and writes to psi issued on other streams must be complete before it.
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
constexpr int kNoAllocStatusInts = 16;  // the SweepStatus block, padded; the level counters follow it
static_assert(sizeof(SweepStatus) <= kNoAllocStatusInts * sizeof(int), "status block overlaps the level counters");
static __device__ __align__(256) int g_noalloc_scratch[kNoAllocStatusInts + kNoAllocMaxLevels];

constexpr int kMaxDevices = 64;
void* g_noalloc_ptr[kMaxDevices] = {};
int g_noalloc_per_sm[kMaxDevices] = {};   // resident dataflow CTAs per SM, per device

}  // namespace
}  // namespace lb

extern "C" int lb_transport_inv_noalloc(lb_handle* hh, float* psi) {
    using namespace lb;
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || !psi) return LB_ERR_ARG;
    if (h->device < 0) return fail(h, LB_ERR_STATE, "host-only handle: no device attached");
    if (!h->mesh_ready || !h->angle_ready || h->sigt.empty())
        return fail(h, LB_ERR_STATE, "TransportOp%MatInv was called, but the operator was not ready.");
    // the sweep reads and writes the four nodes of an element as one 16-byte vector
    if (reinterpret_cast<uintptr_t>(psi) % 16 != 0)
        return fail(h, LB_ERR_ARG, "lb_transport_inv_noalloc: psi must be 16-byte aligned");
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
    SweepArgs a{};
    a.items = h->d_items;
    a.pitems = h->d_pitems;
    a.pbase = h->d_pbase;
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
    int& per_sm = g_noalloc_per_sm[h->device];
    if (per_sm < 1) {
        int n = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sweep_dataflow_kernel, 256, 0);
        per_sm = n < 1 ? 1 : n;
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
