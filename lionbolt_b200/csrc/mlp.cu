// Learned right preconditioner for FGMRES: a per-cell MLP on the flux-moment residual.
//
// No counterpart in the reference (which preconditions only with the sweep, BoltzmannOperator.f90:
// 59-104).  For a moment-space vector v (a Krylov basis vector, i.e. residual-like), the network
// sees per cell e
//   x = ( vbar_j(e) / s_e  for j < 16 (l <= 3),  sigma_t*ell,  sigma_s0*ell,  sigma_s0/sigma_t )
// where vbar_j is the cell average of moment j (the mean of the 4 nodal values of a linear tet),
// s_e = sqrt(mean_j vbar_j^2) its scale and ell = 4V/S the mean chord of the cell (volume over
// surface; the cell volume enters through it).  It predicts o = 16 cell-average corrections and the
// preconditioner returns
//   z = v + s_e * o_j(e)   on the 4 nodes of e for j < 16,      z = v   for j >= 16,
// an approximation of A^{-1} v = v + (A^{-1} - I) v.  Trained on (r, e) pairs with r = A e from
// source-iteration runs of the plain solver: target (ebar - rbar) / s_e.
//
// Network: 19 -> 64 -> 64 -> 16, ReLU, 6,480 parameters.  Weights and activations in BF16 with
// FP32 accumulation (inference on tensor cores with mma.sync m16n8k16, hidden activations kept
// in registers between layers); FP32 master weights, FP32 gradients, Adam.
#include "lb_internal.h"
#include <algorithm>
#include <cmath>
#include <cstring>

namespace lb {

namespace lp {
constexpr int NMOM = 16;
constexpr int NIN = 19;
constexpr int NH = 64;
constexpr int NOUT = 16;
constexpr int OFF_W1 = 0;                    // [64][19]
constexpr int OFF_B1 = OFF_W1 + NH * NIN;    // [64]
constexpr int OFF_W2 = OFF_B1 + NH;          // [64][64]
constexpr int OFF_B2 = OFF_W2 + NH * NH;     // [64]
constexpr int OFF_W3 = OFF_B2 + NH;          // [16][64]
constexpr int OFF_B3 = OFF_W3 + NOUT * NH;   // [16]
constexpr int NPARAM = OFF_B3 + NOUT;        // 6480
constexpr int FS = 20;                       // stored feature stride (floats)
// inference: BF16 weight rows in shared memory, padded so that the B-fragment loads of a warp
// (8 rows x 4 word columns) fall in 32 distinct banks
constexpr int RS1 = 40, RS2 = 72, RS3 = 72, RSX = 40;
constexpr int kWarps = 8;
constexpr int kThreads = kWarps * 32;
// training: FP32 weights in shared memory with odd row strides (conflict-free row and column walks)
constexpr int TS1 = 19, TS2 = 65, TS3 = 65;
constexpr int T_W1 = 0, T_B1 = T_W1 + NH * TS1, T_W2 = T_B1 + NH, T_B2 = T_W2 + NH * TS2, T_W3 = T_B2 + NH,
              T_B3 = T_W3 + NOUT * TS3, T_N = T_B3 + NOUT;
}  // namespace lp

struct MlpState {
    float* d_w = nullptr;          // [NPARAM] FP32 master weights
    float* d_m = nullptr;          // Adam first moment
    float* d_v = nullptr;          // Adam second moment
    float* d_part = nullptr;       // [max_parts][NPARAM] per-block gradient partials
    double* d_lossp = nullptr;     // [max_parts] per-block loss partials
    double* d_losshist = nullptr;  // [hist_cap]
    int max_parts = 0;
    int hist_cap = 0;
    float* d_X = nullptr;          // [cap][FS] sample features
    float* d_T = nullptr;          // [cap][16] sample targets
    long long nsamples = 0, cap = 0;
    float* d_chord = nullptr;      // [NE] mean chord 4V/S
    float2* d_matxs = nullptr;     // [Nm] (sigma_t, sigma_s0) of the current within-group cross sections
    int matxs_version = -1;
    int cell_mesh_version = -1;    // mesh the chord / material tables belong to
    int adam_t = 0;
    bool have_weights = false;
    bool enabled = false;
};

static MlpState* S(Handle* h) { return reinterpret_cast<MlpState*>(h->mlp); }

static MlpState* state(Handle* h) {
    if (!h->mlp) h->mlp = new MlpState();
    return S(h);
}

bool mlp_ready(Handle* h) { return h->mlp && S(h)->have_weights && S(h)->enabled; }

void mlp_destroy(Handle* h) {
    MlpState* s = S(h);
    if (!s) return;
    for (void* p : {(void*)s->d_w, (void*)s->d_m, (void*)s->d_v, (void*)s->d_part, (void*)s->d_lossp,
                    (void*)s->d_losshist, (void*)s->d_X, (void*)s->d_T, (void*)s->d_chord, (void*)s->d_matxs})
        if (p) cudaFree(p);
    delete s;
    h->mlp = nullptr;
}

namespace {

using lp::NPARAM;

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ uint32_t ld32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Shared-memory image of the network for tensor-core inference.
struct InferSmem {
    __nv_bfloat16 w1[lp::NH * lp::RS1];
    __nv_bfloat16 w2[lp::NH * lp::RS2];
    __nv_bfloat16 w3[lp::NOUT * lp::RS3];
    float b1[lp::NH], b2[lp::NH], b3[lp::NOUT];
    __nv_bfloat16 x[lp::kWarps][16 * lp::RSX];   // per-warp feature tile (16 cells)
    float o[lp::kWarps][16 * 17];                // per-warp output tile
    float sc[lp::kWarps][16];                    // per-warp cell scales
};

__device__ void load_infer_weights(InferSmem& sm, const float* __restrict__ w) {
    using namespace lp;
    for (int i = threadIdx.x; i < NH * RS1; i += blockDim.x) {
        const int r = i / RS1, c = i % RS1;
        sm.w1[i] = __float2bfloat16_rn(c < NIN ? w[OFF_W1 + r * NIN + c] : 0.f);
    }
    for (int i = threadIdx.x; i < NH * RS2; i += blockDim.x) {
        const int r = i / RS2, c = i % RS2;
        sm.w2[i] = __float2bfloat16_rn(c < NH ? w[OFF_W2 + r * NH + c] : 0.f);
    }
    for (int i = threadIdx.x; i < NOUT * RS3; i += blockDim.x) {
        const int r = i / RS3, c = i % RS3;
        sm.w3[i] = __float2bfloat16_rn(c < NH ? w[OFF_W3 + r * NH + c] : 0.f);
    }
    for (int i = threadIdx.x; i < NH; i += blockDim.x) {
        sm.b1[i] = w[OFF_B1 + i];
        sm.b2[i] = w[OFF_B2 + i];
    }
    for (int i = threadIdx.x; i < NOUT; i += blockDim.x) sm.b3[i] = w[OFF_B3 + i];
    // zero the padding columns of every feature tile once (features only ever fill columns < 19)
    for (int i = threadIdx.x; i < kWarps * 16 * RSX; i += blockDim.x) (&sm.x[0][0])[i] = __float2bfloat16_rn(0.f);
}

// One warp evaluates the network on the 16 feature rows of sm.x[warp] and leaves the 16 x 16
// outputs in sm.o[warp] (row = cell, column = moment).
__device__ __forceinline__ void mlp_tile(InferSmem& sm, int warp, int lane) {
    using namespace lp;
    const int g = lane >> 2, t = lane & 3;
    const __nv_bfloat16* X = sm.x[warp];
    uint32_t a[4][4];
#pragma unroll
    for (int ks = 0; ks < 2; ++ks) {
        a[ks][0] = ld32(X + g * RSX + ks * 16 + 2 * t);
        a[ks][1] = ld32(X + (g + 8) * RSX + ks * 16 + 2 * t);
        a[ks][2] = ld32(X + g * RSX + ks * 16 + 2 * t + 8);
        a[ks][3] = ld32(X + (g + 8) * RSX + ks * 16 + 2 * t + 8);
    }
    float acc[8][4];
    // layer 1: [16 x 32] x [32 x 64]
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
#pragma unroll
        for (int ks = 0; ks < 2; ++ks) {
            const __nv_bfloat16* wr = sm.w1 + (nt * 8 + g) * RS1 + ks * 16 + 2 * t;
            mma_bf16(acc[nt], a[ks], ld32(wr), ld32(wr + 8));
        }
    }
    // bias + ReLU, rounded to BF16 and repacked as the A operand of the next layer
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
#pragma unroll
        for (int hf = 0; hf < 2; ++hf) {
            const int nt = 2 * kk + hf, c = nt * 8 + 2 * t;
            const float v0 = fmaxf(acc[nt][0] + sm.b1[c], 0.f), v1 = fmaxf(acc[nt][1] + sm.b1[c + 1], 0.f);
            const float v2 = fmaxf(acc[nt][2] + sm.b1[c], 0.f), v3 = fmaxf(acc[nt][3] + sm.b1[c + 1], 0.f);
            a[kk][2 * hf + 0] = pack_bf16(v0, v1);
            a[kk][2 * hf + 1] = pack_bf16(v2, v3);
        }
    }
    // layer 2: [16 x 64] x [64 x 64]
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) {
            const __nv_bfloat16* wr = sm.w2 + (nt * 8 + g) * RS2 + ks * 16 + 2 * t;
            mma_bf16(acc[nt], a[ks], ld32(wr), ld32(wr + 8));
        }
    }
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
#pragma unroll
        for (int hf = 0; hf < 2; ++hf) {
            const int nt = 2 * kk + hf, c = nt * 8 + 2 * t;
            const float v0 = fmaxf(acc[nt][0] + sm.b2[c], 0.f), v1 = fmaxf(acc[nt][1] + sm.b2[c + 1], 0.f);
            const float v2 = fmaxf(acc[nt][2] + sm.b2[c], 0.f), v3 = fmaxf(acc[nt][3] + sm.b2[c + 1], 0.f);
            a[kk][2 * hf + 0] = pack_bf16(v0, v1);
            a[kk][2 * hf + 1] = pack_bf16(v2, v3);
        }
    }
    // layer 3: [16 x 64] x [64 x 16]
    float* O = sm.o[warp];
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) {
        float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) {
            const __nv_bfloat16* wr = sm.w3 + (nt * 8 + g) * RS3 + ks * 16 + 2 * t;
            mma_bf16(d, a[ks], ld32(wr), ld32(wr + 8));
        }
        const int c = nt * 8 + 2 * t;
        O[g * 17 + c] = d[0] + sm.b3[c];
        O[g * 17 + c + 1] = d[1] + sm.b3[c + 1];
        O[(g + 8) * 17 + c] = d[2] + sm.b3[c];
        O[(g + 8) * 17 + c + 1] = d[3] + sm.b3[c + 1];
    }
}

__device__ __forceinline__ void cell_scalars(long long e, const float* __restrict__ chord, const int* __restrict__ mat,
                                             const float2* __restrict__ matxs, float& f0, float& f1, float& f2) {
    const float l = chord[e];
    const float2 xs = matxs[mat[e]];
    f0 = xs.x * l;
    f1 = xs.y * l;
    f2 = xs.x > 0.f ? xs.y / xs.x : 0.f;
}

// z = v + s_e * net(features(v)) lifted to the nodes for j < nmom; z = v for the other moments.
// Moment vectors are FP64 [nm][NENK].  One warp per 16 cells; lane L reads cell L/2, nodes
// 2(L&1), 2(L&1)+1, so each moment row of the tile is one coalesced 512-byte access.
__global__ void __launch_bounds__(lp::kThreads, 2) lp_apply_kernel(const float* __restrict__ w, const double* __restrict__ v,
                                                                  double* __restrict__ z, const float* __restrict__ chord,
                                                                  const int* __restrict__ mat,
                                                                  const float2* __restrict__ matxs, long long NE,
                                                                  long long NENK, int nm, int nmom, double vscale) {
    // vscale: v * vscale is the vector whose features the network sees (an unnormalised Krylov basis
    // vector times its scale); the correction is returned in v's units
    extern __shared__ __align__(16) unsigned char smraw[];
    InferSmem& sm = *reinterpret_cast<InferSmem*>(smraw);
    load_infer_weights(sm, w);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = lane >> 1, hf = lane & 1;
    const long long ntiles = (NE + 15) / 16;
    for (long long tile = (long long)blockIdx.x * lp::kWarps + warp; tile < ntiles;
         tile += (long long)gridDim.x * lp::kWarps) {
        const long long e = tile * 16 + c;
        const bool valid = e < NE;
        const size_t off = (size_t)(4 * e + 2 * hf);
        float avg[lp::NMOM];
        float ss = 0.f;
#pragma unroll
        for (int j = 0; j < lp::NMOM; ++j) {
            double sum = 0.0;
            if (valid && j < nmom) {
                const double2 d = __ldg(reinterpret_cast<const double2*>(v + (size_t)j * NENK + off));
                sum = d.x + d.y;
            }
            sum += __shfl_xor_sync(0xffffffffu, sum, 1);
            avg[j] = (float)(0.25 * vscale * sum);
            ss = fmaf(avg[j], avg[j], ss);
        }
        const float s = sqrtf(ss / (float)nmom);
        const float inv = s > 0.f ? 1.f / s : 0.f;
        __nv_bfloat16* X = sm.x[warp] + c * lp::RSX;
#pragma unroll
        for (int j = 0; j < lp::NMOM; ++j)
            if ((j >> 3) == hf) X[j] = __float2bfloat16_rn(avg[j] * inv);
        if (hf == 0) {
            float f0 = 0.f, f1 = 0.f, f2 = 0.f;
            if (valid) cell_scalars(e, chord, mat, matxs, f0, f1, f2);
            X[16] = __float2bfloat16_rn(f0);
            X[17] = __float2bfloat16_rn(f1);
            X[18] = __float2bfloat16_rn(f2);
            sm.sc[warp][c] = s;
        }
        __syncwarp();
        mlp_tile(sm, warp, lane);
        __syncwarp();
        if (valid) {
            const float* O = sm.o[warp] + c * 17;
            for (int j = 0; j < nm; ++j) {
                const double2 d = __ldg(reinterpret_cast<const double2*>(v + (size_t)j * NENK + off));
                const double corr = j < nmom ? (double)s * (double)O[j] / vscale : 0.0;
                *reinterpret_cast<double2*>(z + (size_t)j * NENK + off) = make_double2(d.x + corr, d.y + corr);
            }
        }
        __syncwarp();
    }
}

// Y[n][16] = net(X[n][0..18]) for explicit features (stride FS).
__global__ void __launch_bounds__(lp::kThreads, 2) lp_forward_kernel(const float* __restrict__ w, const float* __restrict__ X,
                                                                    long long n, float* __restrict__ Y) {
    extern __shared__ __align__(16) unsigned char smraw[];
    InferSmem& sm = *reinterpret_cast<InferSmem*>(smraw);
    load_infer_weights(sm, w);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long ntiles = (n + 15) / 16;
    for (long long tile = (long long)blockIdx.x * lp::kWarps + warp; tile < ntiles;
         tile += (long long)gridDim.x * lp::kWarps) {
        const long long r0 = tile * 16;
        for (int i = lane; i < 16 * lp::NIN; i += 32) {
            const int r = i / lp::NIN, col = i % lp::NIN;
            const float val = r0 + r < n ? X[(r0 + r) * lp::FS + col] : 0.f;
            sm.x[warp][r * lp::RSX + col] = __float2bfloat16_rn(val);
        }
        __syncwarp();
        mlp_tile(sm, warp, lane);
        __syncwarp();
        for (int i = lane; i < 16 * lp::NOUT; i += 32) {
            const int r = i / lp::NOUT, col = i % lp::NOUT;
            if (r0 + r < n) Y[(r0 + r) * lp::NOUT + col] = sm.o[warp][r * 17 + col];
        }
        __syncwarp();
    }
}

// Training samples from a (residual, error) pair of moment vectors: cells drawn by a counter hash.
//   X[o][0..15] = rbar_j / s, X[o][16..18] = cell scalars, T[o][j] = (ebar_j - rbar_j) / s,
//   X[o][19] = s^2 / (mean square of the field's moments j < nmom): the sample's loss weight, so
//   that the loss measures the correction s * o in the field's own units and cells with a
//   vanishing residual (whose scaled targets are unbounded) carry no weight.
__global__ void lp_sample_kernel(const double* __restrict__ r, const double* __restrict__ err, long long NE,
                                 long long NENK, int nmom, const float* __restrict__ chord, const int* __restrict__ mat,
                                 const float2* __restrict__ matxs, unsigned long long seed, long long count,
                                 double inv_ms, float* __restrict__ X, float* __restrict__ T) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= count) return;
    const long long e = (long long)(mix64(seed ^ mix64((unsigned long long)q)) % (unsigned long long)NE);
    double rb[lp::NMOM], eb[lp::NMOM];
    double ss = 0.0;
    for (int j = 0; j < lp::NMOM; ++j) {
        rb[j] = eb[j] = 0.0;
        if (j < nmom) {
            const double* pr = r + (size_t)j * NENK + 4 * e;
            const double* pe = err + (size_t)j * NENK + 4 * e;
            rb[j] = 0.25 * (pr[0] + pr[1] + pr[2] + pr[3]);
            eb[j] = 0.25 * (pe[0] + pe[1] + pe[2] + pe[3]);
        }
        ss += rb[j] * rb[j];
    }
    const double s = sqrt(ss / nmom);
    const double inv = s > 0.0 ? 1.0 / s : 0.0;
    float* x = X + q * lp::FS;
    float* t = T + q * lp::NOUT;
    for (int j = 0; j < lp::NMOM; ++j) {
        x[j] = (float)(rb[j] * inv);
        t[j] = (float)((eb[j] - rb[j]) * inv);
    }
    float f0, f1, f2;
    cell_scalars(e, chord, mat, matxs, f0, f1, f2);
    x[16] = f0;
    x[17] = f1;
    x[18] = f2;
    x[19] = (float)(s * s * inv_ms);   // loss weight: the cell's share of the field's residual
}

// Loss and gradient of L = 1/(2n) sum_samples w sum_i (o_i - t_i)^2 over a batch (w = feature
// column 19), one warp per sample.
// The forward pass rounds weights, inputs and hidden activations to BF16 exactly like the
// inference kernel; the backward pass treats the rounding as identity (straight-through) and
// runs in FP32.  Each block accumulates its gradient in shared memory and writes one partial.
// Samples: direct (s-th sample of the batch is sample s) or drawn by hash(seed, s) % nsamples.
__global__ void __launch_bounds__(lp::kThreads) lp_grad_kernel(const float* __restrict__ w, const float* __restrict__ X,
                                                              const float* __restrict__ T, long long nsamples, int batch,
                                                              int direct, unsigned long long seed, float inv_n,
                                                              float* __restrict__ part, double* __restrict__ lossp) {
    using namespace lp;
    extern __shared__ __align__(16) float smf[];
    float* sw = smf;            // [T_N] BF16-rounded weights (FP32 biases), padded rows
    float* sg = smf + T_N;      // [NPARAM] gradient accumulator (unpadded parameter layout)
    __shared__ double wl[kWarps];
    for (int i = threadIdx.x; i < NH * NIN; i += blockDim.x) sw[T_W1 + (i / NIN) * TS1 + i % NIN] = bf16r(w[OFF_W1 + i]);
    for (int i = threadIdx.x; i < NH * NH; i += blockDim.x) sw[T_W2 + (i / NH) * TS2 + i % NH] = bf16r(w[OFF_W2 + i]);
    for (int i = threadIdx.x; i < NOUT * NH; i += blockDim.x) sw[T_W3 + (i / NH) * TS3 + i % NH] = bf16r(w[OFF_W3 + i]);
    for (int i = threadIdx.x; i < NH; i += blockDim.x) {
        sw[T_B1 + i] = w[OFF_B1 + i];
        sw[T_B2 + i] = w[OFF_B2 + i];
    }
    for (int i = threadIdx.x; i < NOUT; i += blockDim.x) sw[T_B3 + i] = w[OFF_B3 + i];
    for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) sg[i] = 0.f;
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned FULL = 0xffffffffu;
    float loss = 0.f;
    for (int sidx = blockIdx.x * kWarps + warp; sidx < batch; sidx += gridDim.x * kWarps) {
        const long long n = direct ? (long long)sidx
                                   : (long long)(mix64(seed ^ mix64((unsigned long long)sidx)) % (unsigned long long)nsamples);
        const float xk = lane < NIN ? bf16r(X[n * FS + lane]) : 0.f;
        // layer 1 (lane owns hidden units lane, lane+32)
        float z1a = sw[T_B1 + lane], z1b = sw[T_B1 + lane + 32];
#pragma unroll
        for (int k = 0; k < NIN; ++k) {
            const float xb = __shfl_sync(FULL, xk, k);
            z1a = fmaf(sw[T_W1 + lane * TS1 + k], xb, z1a);
            z1b = fmaf(sw[T_W1 + (lane + 32) * TS1 + k], xb, z1b);
        }
        const float h1a = bf16r(fmaxf(z1a, 0.f)), h1b = bf16r(fmaxf(z1b, 0.f));
        // layer 2
        float z2a = sw[T_B2 + lane], z2b = sw[T_B2 + lane + 32];
#pragma unroll 8
        for (int j = 0; j < NH; ++j) {
            const float hb = __shfl_sync(FULL, j < 32 ? h1a : h1b, j & 31);
            z2a = fmaf(sw[T_W2 + lane * TS2 + j], hb, z2a);
            z2b = fmaf(sw[T_W2 + (lane + 32) * TS2 + j], hb, z2b);
        }
        const float h2a = bf16r(fmaxf(z2a, 0.f)), h2b = bf16r(fmaxf(z2b, 0.f));
        // layer 3: lane -> output lane&15 over the half lane>>4 of the hidden units
        const int oi = lane & 15, jh = lane >> 4;
        float o = 0.f;
#pragma unroll 8
        for (int jj = 0; jj < 32; ++jj) {
            const float ha = __shfl_sync(FULL, h2a, jj), hb = __shfl_sync(FULL, h2b, jj);
            o = fmaf(sw[T_W3 + oi * TS3 + jh * 32 + jj], jh ? hb : ha, o);
        }
        o += __shfl_xor_sync(FULL, o, 16);
        o += sw[T_B3 + oi];
        const float wt = X[n * FS + NIN];
        const float diff = o - T[n * NOUT + oi];
        if (lane < 16) loss = fmaf(wt * diff, diff, loss);
        const float d3 = wt * diff * inv_n;   // dL/do_i (lanes i and i+16 hold the same value)
        // output layer gradients
        if (lane < 16) atomicAdd(&sg[OFF_B3 + lane], d3);
        float g2a = 0.f, g2b = 0.f;
#pragma unroll 4
        for (int i = 0; i < NOUT; ++i) {
            const float di = __shfl_sync(FULL, d3, i);
            atomicAdd(&sg[OFF_W3 + i * NH + lane], di * h2a);
            atomicAdd(&sg[OFF_W3 + i * NH + lane + 32], di * h2b);
            g2a = fmaf(sw[T_W3 + i * TS3 + lane], di, g2a);
            g2b = fmaf(sw[T_W3 + i * TS3 + lane + 32], di, g2b);
        }
        const float d2a = z2a > 0.f ? g2a : 0.f, d2b = z2b > 0.f ? g2b : 0.f;
        atomicAdd(&sg[OFF_B2 + lane], d2a);
        atomicAdd(&sg[OFF_B2 + lane + 32], d2b);
        float g1a = 0.f, g1b = 0.f;
        for (int i = 0; i < NH; ++i) {
            const float di = __shfl_sync(FULL, i < 32 ? d2a : d2b, i & 31);
            if (di != 0.f) {
                atomicAdd(&sg[OFF_W2 + i * NH + lane], di * h1a);
                atomicAdd(&sg[OFF_W2 + i * NH + lane + 32], di * h1b);
                g1a = fmaf(sw[T_W2 + i * TS2 + lane], di, g1a);
                g1b = fmaf(sw[T_W2 + i * TS2 + lane + 32], di, g1b);
            }
        }
        const float d1a = z1a > 0.f ? g1a : 0.f, d1b = z1b > 0.f ? g1b : 0.f;
        atomicAdd(&sg[OFF_B1 + lane], d1a);
        atomicAdd(&sg[OFF_B1 + lane + 32], d1b);
        for (int i = 0; i < NH; ++i) {
            const float di = __shfl_sync(FULL, i < 32 ? d1a : d1b, i & 31);
            if (di != 0.f && lane < NIN) atomicAdd(&sg[OFF_W1 + i * NIN + lane], di * xk);
        }
    }
    // block loss
    for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(FULL, loss, o);
    if (lane == 0) wl[warp] = (double)loss;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < kWarps; ++k) s += wl[k];
        lossp[blockIdx.x] = 0.5 * s * (double)inv_n;
    }
    for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) part[(size_t)blockIdx.x * NPARAM + i] = sg[i];
}

// Sum of the block partials in block order (deterministic) and one Adam step; block 0 thread 0
// also records the batch loss.
__global__ void lp_adam_kernel(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                               const float* __restrict__ part, const double* __restrict__ lossp, int nparts, float lr,
                               float beta1, float beta2, float eps, float bc1, float bc2, double* __restrict__ losshist,
                               int step) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p == 0 && losshist) {
        double s = 0.0;
        for (int b = 0; b < nparts; ++b) s += lossp[b];
        losshist[step] = s;
    }
    if (p >= NPARAM) return;
    float g = 0.f;
    for (int b = 0; b < nparts; ++b) g += part[(size_t)b * NPARAM + p];
    const float mm = beta1 * m[p] + (1.f - beta1) * g;
    const float vv = beta2 * v[p] + (1.f - beta2) * g * g;
    m[p] = mm;
    v[p] = vv;
    w[p] -= lr * (mm / bc1) / (sqrtf(vv / bc2) + eps);
}

// Gradient sum without an update (gradient checks).
__global__ void lp_gradsum_kernel(const float* __restrict__ part, int nparts, float* __restrict__ g) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= NPARAM) return;
    float s = 0.f;
    for (int b = 0; b < nparts; ++b) s += part[(size_t)b * NPARAM + p];
    g[p] = s;
}

constexpr size_t kGradSmem = sizeof(float) * (lp::T_N + lp::NPARAM);

}  // namespace

// ---------------------------------------------------------------------------------------------
//  host side
// ---------------------------------------------------------------------------------------------
static int ensure_weights_buf(Handle* h, MlpState* s) {
    if (s->d_w) return LB_OK;
    cudaError_t e = cudaMalloc(&s->d_w, sizeof(float) * NPARAM);
    if (e == cudaSuccess) e = cudaMalloc(&s->d_m, sizeof(float) * NPARAM);
    if (e == cudaSuccess) e = cudaMalloc(&s->d_v, sizeof(float) * NPARAM);
    if (e != cudaSuccess) return cuda_fail(h, e, "network weights");
    return LB_OK;
}

static int reset_adam(Handle* h, MlpState* s) {
    cudaError_t e = cudaMemsetAsync(s->d_m, 0, sizeof(float) * NPARAM, h->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->d_v, 0, sizeof(float) * NPARAM, h->stream);
    s->adam_t = 0;
    return e == cudaSuccess ? LB_OK : cuda_fail(h, e, "reset optimiser");
}

// Per-cell mean chord and the per-material (sigma_t, sigma_s0) table of the current cross sections.
static int ensure_cell_data(Handle* h, MlpState* s) {
    cudaError_t e = cudaSuccess;
    if (s->cell_mesh_version != h->mesh_version) {
        if (s->d_chord) cudaFree(s->d_chord);
        if (s->d_matxs) cudaFree(s->d_matxs);
        s->d_chord = nullptr;
        s->d_matxs = nullptr;
        s->cell_mesh_version = h->mesh_version;
    }
    if (!s->d_chord) {
        std::vector<float> ch(h->NE);
        for (int el = 0; el < h->NE; ++el) {
            double S = 0.0;   // sum_f A_f / V
            for (int f = 0; f < 4; ++f) {
                const double* sv = &h->svec[(size_t)el * 12 + f * 3];
                S += std::sqrt(sv[0] * sv[0] + sv[1] * sv[1] + sv[2] * sv[2]);
            }
            ch[el] = (float)(4.0 / S);
        }
        e = cudaMalloc(&s->d_chord, sizeof(float) * h->NE);
        if (e == cudaSuccess) e = cudaMemcpy(s->d_chord, ch.data(), sizeof(float) * h->NE, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return cuda_fail(h, e, "cell chords");
    }
    if (!s->d_matxs) {
        e = cudaMalloc(&s->d_matxs, sizeof(float2) * std::max(h->Nm, 1));
        if (e != cudaSuccess) return cuda_fail(h, e, "material table");
        s->matxs_version = -1;
    }
    if (s->matxs_version != h->xs_version) {
        std::vector<float2> t(h->Nm);
        const int Lp1 = h->Ls + 1;
        for (int m = 0; m < h->Nm; ++m) t[m] = make_float2((float)h->sigt[m], (float)h->sigs[(size_t)m * Lp1]);
        e = cudaMemcpyAsync(s->d_matxs, t.data(), sizeof(float2) * h->Nm, cudaMemcpyHostToDevice, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) return cuda_fail(h, e, "material table");
        s->matxs_version = h->xs_version;
    }
    return LB_OK;
}

static int infer_grid(Handle* h, const void* kernel, long long ntiles) {
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, lp::kThreads, sizeof(InferSmem));
    cudaGetLastError();
    per_sm = std::max(per_sm, 1);
    const long long blocks = (ntiles + lp::kWarps - 1) / lp::kWarps;
    return (int)std::max<long long>(1, std::min<long long>(blocks, (long long)h->sm_count * per_sm));
}

int mlp_apply_precond(Handle* h, const double* v, double* z, double vscale) {
    MlpState* s = S(h);
    if (!s || !s->have_weights) return fail(h, LB_ERR_STATE, "learned preconditioner: no weights loaded");
    int rc = ensure_cell_data(h, s);
    if (rc) return rc;
    const long long ntiles = ((long long)h->NE + 15) / 16;
    const int grid = infer_grid(h, (const void*)lp_apply_kernel, ntiles);
    Timer t;
    timer_begin(h, LB_T_PRECOND, t);
    lp_apply_kernel<<<grid, lp::kThreads, sizeof(InferSmem), h->stream>>>(
        s->d_w, v, z, s->d_chord, h->d_mat, s->d_matxs, (long long)h->NE, h->NENK, h->nm, std::min(h->nm, lp::NMOM),
        vscale);
    cudaError_t e = cudaGetLastError();
    timer_end(h, t);
    return e == cudaSuccess ? LB_OK : cuda_fail(h, e, "preconditioner kernel");
}

int mlp_sample(Handle* h, const double* r, const double* err, long long count, unsigned long long seed) {
    MlpState* s = state(h);
    int rc = ensure_cell_data(h, s);
    if (rc) return rc;
    if (count <= 0) return LB_OK;
    if (s->nsamples + count > s->cap) {
        long long ncap = std::max<long long>(2 * s->cap, s->nsamples + count);
        float *nx = nullptr, *nt = nullptr;
        cudaError_t e = cudaMalloc(&nx, sizeof(float) * lp::FS * ncap);
        if (e == cudaSuccess) e = cudaMalloc(&nt, sizeof(float) * lp::NOUT * ncap);
        if (e != cudaSuccess) {
            if (nx) cudaFree(nx);
            return cuda_fail(h, e, "training samples");
        }
        if (s->nsamples) {
            cudaMemcpyAsync(nx, s->d_X, sizeof(float) * lp::FS * s->nsamples, cudaMemcpyDeviceToDevice, h->stream);
            cudaMemcpyAsync(nt, s->d_T, sizeof(float) * lp::NOUT * s->nsamples, cudaMemcpyDeviceToDevice, h->stream);
        }
        cudaStreamSynchronize(h->stream);
        if (s->d_X) cudaFree(s->d_X);
        if (s->d_T) cudaFree(s->d_T);
        s->d_X = nx;
        s->d_T = nt;
        s->cap = ncap;
    }
    // mean square of the moments the network sees (nodal values; a per-field constant)
    const int nmom = std::min(h->nm, lp::NMOM);
    const size_t nn = (size_t)nmom * (size_t)h->NENK;
    double ss = 0.0;
    if ((rc = k_dots(h, r, nn, 1, r, nn, &ss))) return rc;
    const double inv_ms = ss > 0.0 ? (double)nn / ss : 0.0;
    const int tpb = 128;
    lp_sample_kernel<<<(unsigned)((count + tpb - 1) / tpb), tpb, 0, h->stream>>>(
        r, err, (long long)h->NE, h->NENK, nmom, s->d_chord, h->d_mat, s->d_matxs, seed, count, inv_ms,
        s->d_X + (size_t)lp::FS * s->nsamples, s->d_T + (size_t)lp::NOUT * s->nsamples);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(h, e, "sample kernel");
    s->nsamples += count;
    return LB_OK;
}

static int ensure_grad_bufs(Handle* h, MlpState* s, int parts, int hist) {
    cudaError_t e = cudaSuccess;
    if (parts > s->max_parts) {
        if (s->d_part) cudaFree(s->d_part);
        if (s->d_lossp) cudaFree(s->d_lossp);
        s->d_part = nullptr;
        s->d_lossp = nullptr;
        e = cudaMalloc(&s->d_part, sizeof(float) * NPARAM * (size_t)parts);
        if (e == cudaSuccess) e = cudaMalloc(&s->d_lossp, sizeof(double) * parts);
        if (e != cudaSuccess) return cuda_fail(h, e, "gradient partials");
        s->max_parts = parts;
    }
    if (hist > s->hist_cap) {
        if (s->d_losshist) cudaFree(s->d_losshist);
        e = cudaMalloc(&s->d_losshist, sizeof(double) * hist);
        if (e != cudaSuccess) return cuda_fail(h, e, "loss history");
        s->hist_cap = hist;
    }
    static PerDevice attr;
    attr.get([&] {
        cudaFuncSetAttribute(lp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGradSmem);
        cudaGetLastError();
        return 1;
    });
    return LB_OK;
}

// About 8 samples per warp: enough work per block to amortise the weight staging, few enough
// partials for the deterministic block-order reduction.
static int grad_blocks(Handle* h, int batch) {
    return std::max(1, std::min((batch + 8 * lp::kWarps - 1) / (8 * lp::kWarps), h->sm_count));
}

}  // namespace lb

using namespace lb;
struct lb_handle : public lb::Handle {};

namespace {
int need_device(lb_handle* h) {
    if (!h) return LB_ERR_ARG;
    if (h->device < 0) return fail(h, LB_ERR_STATE, "host-only handle: no device attached");
    cudaSetDevice(h->device);
    return LB_OK;
}

// Deterministic uniform(-1, 1) stream for weight initialisation.
struct InitRng {
    unsigned long long x;
    double next() {
        x += 0x9E3779B97F4A7C15ull;
        unsigned long long z = x;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return 2.0 * ((double)(z >> 11) * (1.0 / 9007199254740992.0)) - 1.0;
    }
};
}  // namespace

extern "C" {

int lb_lp_nparams(void) { return lp::NPARAM; }

int lb_lp_init(lb_handle* h, unsigned long long seed) {
    int rc = need_device(h);
    if (rc) return rc;
    MlpState* s = state(h);
    if ((rc = ensure_weights_buf(h, s))) return rc;
    // He-uniform hidden layers; the output layer starts 10x smaller so that the untrained
    // preconditioner is close to the identity.
    std::vector<float> w(lp::NPARAM, 0.f);
    InitRng g{seed};
    const double a1 = std::sqrt(6.0 / lp::NIN), a2 = std::sqrt(6.0 / lp::NH), a3 = 0.1 * std::sqrt(6.0 / (lp::NH + lp::NOUT));
    for (int i = 0; i < lp::NH * lp::NIN; ++i) w[lp::OFF_W1 + i] = (float)(a1 * g.next());
    for (int i = 0; i < lp::NH * lp::NH; ++i) w[lp::OFF_W2 + i] = (float)(a2 * g.next());
    for (int i = 0; i < lp::NOUT * lp::NH; ++i) w[lp::OFF_W3 + i] = (float)(a3 * g.next());
    cudaError_t e = cudaMemcpy(s->d_w, w.data(), sizeof(float) * lp::NPARAM, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(h, e, "upload weights");
    s->have_weights = true;
    s->enabled = true;
    return reset_adam(h, s);
}

int lb_lp_set_weights(lb_handle* h, const float* w) {
    int rc = need_device(h);
    if (rc) return rc;
    if (!w) return fail(h, LB_ERR_ARG, "lb_lp_set_weights: null weights");
    for (int i = 0; i < lp::NPARAM; ++i)
        if (!std::isfinite(w[i])) return fail(h, LB_ERR_NAN, "lb_lp_set_weights: non-finite weight");
    MlpState* s = state(h);
    if ((rc = ensure_weights_buf(h, s))) return rc;
    cudaError_t e = cudaMemcpy(s->d_w, w, sizeof(float) * lp::NPARAM, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(h, e, "upload weights");
    s->have_weights = true;
    s->enabled = true;
    return reset_adam(h, s);
}

int lb_lp_get_weights(lb_handle* h, float* w) {
    int rc = need_device(h);
    if (rc) return rc;
    MlpState* s = S(h);
    if (!w) return fail(h, LB_ERR_ARG, "lb_lp_get_weights: null buffer");
    if (!s || !s->have_weights) return fail(h, LB_ERR_STATE, "lb_lp_get_weights: no weights");
    cudaStreamSynchronize(h->stream);
    cudaError_t e = cudaMemcpy(w, s->d_w, sizeof(float) * lp::NPARAM, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? LB_OK : cuda_fail(h, e, "download weights");
}

int lb_lp_enable(lb_handle* h, int on) {
    int rc = need_device(h);
    if (rc) return rc;
    MlpState* s = state(h);
    if (on && !s->have_weights) return fail(h, LB_ERR_STATE, "lb_lp_enable: no weights loaded");
    s->enabled = on != 0;
    return LB_OK;
}

int lb_lp_forward(lb_handle* h, int n, const float* x, float* y) {
    int rc = need_device(h);
    if (rc) return rc;
    MlpState* s = S(h);
    if (!s || !s->have_weights) return fail(h, LB_ERR_STATE, "lb_lp_forward: no weights");
    if (n < 0 || (n > 0 && (!x || !y))) return fail(h, LB_ERR_ARG, "lb_lp_forward: bad arguments");
    if (n == 0) return LB_OK;
    std::vector<float> xs((size_t)n * lp::FS, 0.f);
    for (int i = 0; i < n; ++i) std::memcpy(&xs[(size_t)i * lp::FS], x + (size_t)i * lp::NIN, sizeof(float) * lp::NIN);
    float *dx = nullptr, *dy = nullptr;
    cudaError_t e = cudaMalloc(&dx, sizeof(float) * xs.size());
    if (e == cudaSuccess) e = cudaMalloc(&dy, sizeof(float) * (size_t)n * lp::NOUT);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dx, xs.data(), sizeof(float) * xs.size(), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) {
        const long long ntiles = ((long long)n + 15) / 16;
        lp_forward_kernel<<<infer_grid(h, (const void*)lp_forward_kernel, ntiles), lp::kThreads, sizeof(InferSmem),
                            h->stream>>>(s->d_w, dx, n, dy);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(y, dy, sizeof(float) * (size_t)n * lp::NOUT, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (dx) cudaFree(dx);
    if (dy) cudaFree(dy);
    return e == cudaSuccess ? LB_OK : cuda_fail(h, e, "lb_lp_forward");
}

int lb_lp_apply(lb_handle* h, const double* v, double* z) {
    int rc = need_device(h);
    if (rc) return rc;
    if (!v || !z) return fail(h, LB_ERR_ARG, "lb_lp_apply: null vector");
    if (!h->phys_ready) return fail(h, LB_ERR_STATE, "lb_lp_apply: cross sections not set");
    const size_t n = (size_t)h->nm * (size_t)h->NENK;
    double *dv = nullptr, *dz = nullptr;
    cudaError_t e = cudaMalloc(&dv, sizeof(double) * n);
    if (e == cudaSuccess) e = cudaMalloc(&dz, sizeof(double) * n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dv, v, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream);
    if (e != cudaSuccess) {
        if (dv) cudaFree(dv);
        if (dz) cudaFree(dz);
        return cuda_fail(h, e, "lb_lp_apply buffers");
    }
    rc = mlp_apply_precond(h, dv, dz, 1.0);
    if (!rc) {
        e = cudaMemcpyAsync(z, dz, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) rc = cuda_fail(h, e, "lb_lp_apply");
    }
    cudaFree(dv);
    cudaFree(dz);
    return rc;
}

int lb_lp_loss_grad(lb_handle* h, int n, const float* x, const float* t, const float* wts, double* loss, float* grad) {
    int rc = need_device(h);
    if (rc) return rc;
    MlpState* s = S(h);
    if (!s || !s->have_weights) return fail(h, LB_ERR_STATE, "lb_lp_loss_grad: no weights");
    if (n <= 0 || !x || !t) return fail(h, LB_ERR_ARG, "lb_lp_loss_grad: bad arguments");
    const int parts = grad_blocks(h, n);
    if ((rc = ensure_grad_bufs(h, s, parts, 1))) return rc;
    std::vector<float> xs((size_t)n * lp::FS, 0.f);
    for (int i = 0; i < n; ++i) {
        std::memcpy(&xs[(size_t)i * lp::FS], x + (size_t)i * lp::NIN, sizeof(float) * lp::NIN);
        xs[(size_t)i * lp::FS + lp::NIN] = wts ? wts[i] : 1.f;
    }
    float *dx = nullptr, *dt = nullptr, *dg = nullptr;
    cudaError_t e = cudaMalloc(&dx, sizeof(float) * xs.size());
    if (e == cudaSuccess) e = cudaMalloc(&dt, sizeof(float) * (size_t)n * lp::NOUT);
    if (e == cudaSuccess) e = cudaMalloc(&dg, sizeof(float) * lp::NPARAM);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dx, xs.data(), sizeof(float) * xs.size(), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dt, t, sizeof(float) * (size_t)n * lp::NOUT, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) {
        lp_grad_kernel<<<parts, lp::kThreads, kGradSmem, h->stream>>>(s->d_w, dx, dt, n, n, 1, 0ull, 1.f / n, s->d_part,
                                                                       s->d_lossp);
        lp_gradsum_kernel<<<(lp::NPARAM + 255) / 256, 256, 0, h->stream>>>(s->d_part, parts, dg);
        e = cudaGetLastError();
    }
    std::vector<double> lp_(parts);
    if (e == cudaSuccess && grad) e = cudaMemcpyAsync(grad, dg, sizeof(float) * lp::NPARAM, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(lp_.data(), s->d_lossp, sizeof(double) * parts, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (dx) cudaFree(dx);
    if (dt) cudaFree(dt);
    if (dg) cudaFree(dg);
    if (e != cudaSuccess) return cuda_fail(h, e, "lb_lp_loss_grad");
    if (loss) {
        double sum = 0.0;
        for (double v : lp_) sum += v;
        *loss = sum;
    }
    return LB_OK;
}

int lb_lp_num_samples(lb_handle* h, long long* n) {
    if (!h || !n) return LB_ERR_ARG;
    *n = h->mlp ? S(h)->nsamples : 0;
    return LB_OK;
}

int lb_lp_get_samples(lb_handle* h, float* x, float* t, float* wts) {
    int rc = need_device(h);
    if (rc) return rc;
    MlpState* s = S(h);
    if (!s || s->nsamples == 0) return LB_OK;
    std::vector<float> xs((size_t)s->nsamples * lp::FS);
    cudaStreamSynchronize(h->stream);
    cudaError_t e = cudaMemcpy(xs.data(), s->d_X, sizeof(float) * xs.size(), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && t) e = cudaMemcpy(t, s->d_T, sizeof(float) * lp::NOUT * s->nsamples, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(h, e, "lb_lp_get_samples");
    for (long long i = 0; i < s->nsamples; ++i) {
        if (x) std::memcpy(x + i * lp::NIN, &xs[(size_t)i * lp::FS], sizeof(float) * lp::NIN);
        if (wts) wts[i] = xs[(size_t)i * lp::FS + lp::NIN];
    }
    return LB_OK;
}

int lb_lp_clear_samples(lb_handle* h) {
    if (!h) return LB_ERR_ARG;
    if (h->mlp) S(h)->nsamples = 0;
    return LB_OK;
}

int lb_lp_train(lb_handle* h, int steps, int batch, double lr, unsigned long long seed, double* loss_hist) {
    int rc = need_device(h);
    if (rc) return rc;
    MlpState* s = S(h);
    if (!s || !s->have_weights) return fail(h, LB_ERR_STATE, "lb_lp_train: no weights (call lb_lp_init)");
    if (s->nsamples <= 0) return fail(h, LB_ERR_STATE, "lb_lp_train: no training samples");
    if (steps < 0 || batch < 1 || !(lr > 0.0)) return fail(h, LB_ERR_ARG, "lb_lp_train: bad arguments");
    const int parts = grad_blocks(h, batch);
    if ((rc = ensure_grad_bufs(h, s, parts, std::max(steps, 1)))) return rc;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const double pi = 3.14159265358979323846;
    for (int it = 0; it < steps; ++it) {
        ++s->adam_t;
        // cosine decay from lr to lr/20
        const double frac = steps > 1 ? (double)it / (double)(steps - 1) : 1.0;
        const float lr_t = (float)(lr * (0.05 + 0.95 * 0.5 * (1.0 + std::cos(pi * frac))));
        const float bc1 = 1.f - std::pow(b1, (float)s->adam_t), bc2 = 1.f - std::pow(b2, (float)s->adam_t);
        lp_grad_kernel<<<parts, lp::kThreads, kGradSmem, h->stream>>>(
            s->d_w, s->d_X, s->d_T, s->nsamples, batch, 0, seed + 0x100000001B3ull * (unsigned long long)it,
            1.f / batch, s->d_part, s->d_lossp);
        lp_adam_kernel<<<(lp::NPARAM + 255) / 256, 256, 0, h->stream>>>(s->d_w, s->d_m, s->d_v, s->d_part, s->d_lossp,
                                                                         parts, lr_t, b1, b2, eps, bc1, bc2,
                                                                         s->d_losshist, it);
    }
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && loss_hist && steps > 0)
        e = cudaMemcpyAsync(loss_hist, s->d_losshist, sizeof(double) * steps, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "lb_lp_train");
    return LB_OK;
}

}  // extern "C"
