// Host side of the B200 transport-solve library: handle management, mesh post-processing,
// quadrature, real spherical harmonics, the per-direction wavefront schedule, and the simple
// C-ABI entry points.  Compiled with -ffp-contract=off: the FP64 face-orientation tests must
// round exactly like the reference's DOT_PRODUCT so that the sweep levels are bit-identical.
#include "lb_internal.h"
#include "gmres_host.h"
#include <algorithm>
#include <cmath>
#include <cstring>
#include <omp.h>
#include <functional>
#include <unordered_map>

namespace lb {

constexpr double PI = 3.14159265358979323846264338327950288;
constexpr double EPS64 = 2.220446049250313080847263336181640625e-16;   // EPSILON(1d0)
constexpr int F2K[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};  // gmsh tet faces

int fail(Handle* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    return code;
}

int cuda_fail(Handle* h, cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    return fail(h, e == cudaErrorMemoryAllocation ? LB_ERR_OOM : LB_ERR_CUDA, m);
}

static double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

static void cross3(const double* a, const double* b, double* c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

// Euclidean norm with the overflow-safe scaling gfortran applies to NORM2.
static double norm3(const double* x) {
    double scale = 0.0, ssq = 1.0;
    for (int i = 0; i < 3; ++i) {
        if (x[i] == 0.0) continue;
        double a = std::fabs(x[i]);
        if (scale < a) { double r = scale / a; ssq = 1.0 + ssq * r * r; scale = a; }
        else { double r = a / scale; ssq += r * r; }
    }
    return scale * std::sqrt(ssq);
}

// Real orthonormal spherical harmonics up to degree Ls at unit direction dir.
// Index j = l*l + l + m, m = -l..l; cos(m phi) for m > 0, sin(|m| phi) for m < 0.
void real_sh(int Ls, const double* dir, double* Y) {
    const double ct = dir[2];
    const double st = std::sqrt(std::max(0.0, 1.0 - ct * ct));
    const double phi = std::atan2(dir[1], dir[0]);
    std::vector<double> P((size_t)(Ls + 1) * (Ls + 1), 0.0);
    auto at = [&](int l, int m) -> double& { return P[(size_t)l * (Ls + 1) + m]; };
    at(0, 0) = 1.0;
    for (int m = 1; m <= Ls; ++m) at(m, m) = at(m - 1, m - 1) * (2.0 * m - 1.0) * st;
    for (int m = 0; m < Ls; ++m) at(m + 1, m) = (2.0 * m + 1.0) * ct * at(m, m);
    for (int m = 0; m <= Ls; ++m)
        for (int l = m + 2; l <= Ls; ++l)
            at(l, m) = ((2.0 * l - 1.0) * ct * at(l - 1, m) - (l + m - 1.0) * at(l - 2, m)) / (l - m);
    for (int l = 0; l <= Ls; ++l)
        for (int m = -l; m <= l; ++m) {
            int am = m < 0 ? -m : m;
            double ratio = 1.0;
            for (int q = l - am + 1; q <= l + am; ++q) ratio /= q;
            double nrm = std::sqrt((2.0 * l + 1.0) / (4.0 * PI) * ratio);
            double v = nrm * at(l, am);
            if (m > 0) v *= std::sqrt(2.0) * std::cos(am * phi);
            if (m < 0) v *= std::sqrt(2.0) * std::sin(am * phi);
            Y[l * l + l + m] = v;
        }
}

void timer_begin(Handle* h, int kind, Timer& t) {
    t.kind = kind;
    if (!h->timing) { t.a = t.b = nullptr; return; }
    if (!h->free_timers.empty()) { t = h->free_timers.back(); h->free_timers.pop_back(); t.kind = kind; }
    else { cudaEventCreate(&t.a); cudaEventCreate(&t.b); }
    cudaEventRecord(t.a, h->stream);
}

void timer_end(Handle* h, Timer& t) {
    h->launches[t.kind] += 1;
    if (!t.a) return;
    cudaEventRecord(t.b, h->stream);
    h->timers.push_back(t);
}

void timers_flush(Handle* h) {
    if (h->timers.empty()) return;
    cudaStreamSynchronize(h->stream);
    for (auto& t : h->timers) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, t.a, t.b) == cudaSuccess) h->acc_ms[t.kind] += ms;
        h->free_timers.push_back(t);
    }
    h->timers.clear();
}

template <class T>
static int dev_alloc(Handle* h, T** p, size_t count, const char* what) {
    if (h->device < 0) return LB_OK;   // host-only handle: schedule and geometry are built, nothing is uploaded
    if (*p) { cudaFree(*p); *p = nullptr; }
    if (count == 0) return LB_OK;
    cudaError_t e = cudaMalloc((void**)p, sizeof(T) * count);
    if (e != cudaSuccess) { *p = nullptr; return cuda_fail(h, e, what); }
    return LB_OK;
}

template <class T>
static int dev_upload(Handle* h, T** p, const T* src, size_t count, const char* what) {
    if (h->device < 0) return LB_OK;
    int rc = dev_alloc(h, p, count, what);
    if (rc) return rc;
    if (count == 0) return LB_OK;
    cudaError_t e = cudaMemcpyAsync(*p, src, sizeof(T) * count, cudaMemcpyHostToDevice, h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, what);
    e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, what);
    return LB_OK;
}

static void free_all(Handle* h) {
    void* ptrs[] = {h->d_geom, h->d_rec, h->d_crec, h->d_crec_base, h->d_blk_elem, h->d_beam_plane, h->d_beam_xyz,
                    h->d_beam_node, h->d_beam_nbr, h->d_cl_start, h->d_cl_base, h->d_ncl, h->d_gtab, h->d_tmat, h->d_mat, h->d_items, h->d_groups, h->d_pitems, h->d_pbase, h->d_chunks, h->d_lvl_start, h->d_lvl_base, h->d_nlev, h->d_done, h->d_status, h->d_tc_err, h->d_dirs, h->d_sigt,
                    h->d_psi, h->d_qext, h->d_Ym2d, h->d_Yd2m, h->d_sigl, h->d_lofj, h->d_V, h->d_Z, h->d_x,
                    h->d_b, h->d_t, h->d_red, h->d_unc, h->d_phi_all, h->d_src, h->d_dose, h->d_flux,
                    h->d_sigl_mg, h->d_yb, h->d_dd};
    for (void* p : ptrs) if (p) cudaFree(p);
    if (h->h_red) cudaFreeHost(h->h_red);
    if (h->d_seg) cudaFree(h->d_seg);
    if (h->h_seg) cudaFreeHost(h->h_seg);
    for (auto& t : h->timers) { cudaEventDestroy(t.a); cudaEventDestroy(t.b); }
    for (auto& t : h->free_timers) { cudaEventDestroy(t.a); cudaEventDestroy(t.b); }
    for (auto& m : h->marks) if (m) cudaEventDestroy(m);
}

// ----------------------------------------------------------------------------------------------
//  Wavefront levels of one direction: the ascending list of elements whose pending upstream
//  faces are all released, level by level.  Each level equals the set the reference's rescanning
//  loop (SweepOrder.f90:137-185) collects, because an element becomes ready exactly when its last
//  upstream neighbour is released, and the reference releases neighbours only after a level is
//  complete.  Cost O(NE log NE) instead of O(levels * NE).
// ----------------------------------------------------------------------------------------------
static bool build_direction(const Handle* h, int i, int* items, std::vector<int>& starts, long long& nz) {
    const int NE = h->NE;
    const double* kv = &h->k[(size_t)i * 3];
    std::vector<uint8_t> upm(NE, 0), outm(NE, 0), cnt(NE, 0);
    std::vector<int> cur, nxt;
    cur.reserve(1024); nxt.reserve(1024);
    nz = 0;
    for (int e = 0; e < NE; ++e) {
        uint8_t u = 0, o = 0;
        for (int f = 0; f < 4; ++f) {
            double kdotn = dot3(kv, &h->nrm[(size_t)e * 12 + f * 3]);
            if (h->nbr[(size_t)e * 4 + f] >= 0 && kdotn < -EPS64) u |= (uint8_t)(1u << f);   // IsUpstream
            if (!(kdotn < 0.0)) o |= (uint8_t)(1u << f);   // outflow term, TransportAlgebra.f90:148-152
        }
        upm[e] = u; outm[e] = o;
        cnt[e] = (uint8_t)__builtin_popcount(u);
        nz += cnt[e];
        if (cnt[e] == 0) cur.push_back(e);
    }
    starts.clear();
    int es = 0;
    while (!cur.empty()) {
        starts.push_back(es);
        for (int e : cur) items[es++] = e | ((int)upm[e] << 24) | ((int)outm[e] << 28);
        nxt.clear();
        for (int e : cur)
            for (int f = 0; f < 4; ++f) {
                int ep = h->nbr[(size_t)e * 4 + f];
                if (ep < 0) continue;
                // local face of ep that faces e (first match, as FINDLOC in SweepOrder.f90:169)
                for (int q = 0; q < 4; ++q)
                    if (h->nbr[(size_t)ep * 4 + q] == e) {
                        if ((upm[ep] >> q) & 1u) { if (--cnt[ep] == 0) nxt.push_back(ep); }
                        break;
                    }
            }
        std::sort(nxt.begin(), nxt.end());
        cur.swap(nxt);
    }
    starts.push_back(es);
    return es == NE;
}

}  // namespace lb

using namespace lb;

struct lb_handle : public lb::Handle {};

extern "C" {

int lb_version(void) { return 10000; }

const char* lb_status_string(int s) {
    switch (s) {
        case LB_OK: return "ok";
        case LB_ERR_ARG: return "invalid argument";
        case LB_ERR_CUDA: return "CUDA error";
        case LB_ERR_OOM: return "out of device memory";
        case LB_ERR_CYCLE: return "sweep is stagnant (cyclic dependency)";
        case LB_ERR_TIMEOUT: return "device dependency wait timed out";
        case LB_ERR_NOCONV: return "iteration did not converge in the iteration limit";
        case LB_ERR_NAN: return "residual norm is NaN";
        case LB_ERR_STATE: return "operator not ready";
        case LB_ERR_BREAKDOWN: return "Krylov breakdown";
        default: return "unknown status";
    }
}

int lb_create(int device, lb_handle** out) {
    if (!out) return LB_ERR_ARG;
    *out = nullptr;
    if (device == -1) {
        // host-only handle: mesh post-processing and sweep scheduling without a GPU
        lb_handle* h = new lb_handle();
        h->device = -1;
        *out = h;
        return LB_OK;
    }
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) return LB_ERR_CUDA;
    if (device < 0 || device >= ndev) return LB_ERR_ARG;
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return LB_ERR_CUDA;
    lb_handle* h = new lb_handle();
    h->device = device;
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) { delete h; return LB_ERR_CUDA; }
    cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (cudaMalloc(&h->d_status, sizeof(SweepStatus)) != cudaSuccess) { delete h; return LB_ERR_OOM; }
    if (cudaMalloc(&h->d_tc_err, sizeof(int)) != cudaSuccess || cudaMemset(h->d_tc_err, 0, sizeof(int)) != cudaSuccess) {
        delete h;
        return LB_ERR_OOM;
    }
    if (cudaMallocHost(&h->h_red, sizeof(double) * 65536) != cudaSuccess) { delete h; return LB_ERR_OOM; }
    if (cudaMalloc(&h->d_red, sizeof(double) * 65536) != cudaSuccess) { delete h; return LB_ERR_OOM; }
    *out = h;
    return LB_OK;
}

int lb_destroy(lb_handle* h) {
    if (!h) return LB_OK;
    if (h->device < 0) { delete h; return LB_OK; }
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->stream);
    free_all(h);
    if (h->mlp) mlp_destroy(h);
    cudaStreamDestroy(h->stream);
    delete h;
    return LB_OK;
}

int lb_last_error(const lb_handle* h, char* buf, int len) {
    if (!buf || len <= 0) return LB_ERR_ARG;
    const char* m = h ? h->err.c_str() : "";
    std::strncpy(buf, m, (size_t)len - 1);
    buf[len - 1] = '\0';
    return LB_OK;
}

int lb_sn_quadrature(int Ng, int Nc, double* k, double* w) {
    if (Ng < 1 || Nc < 1 || !k || !w) return LB_ERR_ARG;
    // Gauss-Legendre by Newton iteration on P_Ng, ascending nodes
    std::vector<double> mu(Ng), wg(Ng);
    for (int i = 0; i < Ng; ++i) {
        double z = std::cos(PI * (i + 0.75) / (Ng + 0.5)), p0 = 1, p1 = z, dp = 1;
        for (int it = 0; it < 100; ++it) {
            p0 = 1.0; p1 = z;
            for (int l = 2; l <= Ng; ++l) { double p2 = ((2.0 * l - 1.0) * z * p1 - (l - 1.0) * p0) / l; p0 = p1; p1 = p2; }
            dp = Ng * (z * p1 - p0) / (z * z - 1.0);
            double dz = p1 / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-16) break;
        }
        p0 = 1.0; p1 = z;
        for (int l = 2; l <= Ng; ++l) { double p2 = ((2.0 * l - 1.0) * z * p1 - (l - 1.0) * p0) / l; p0 = p1; p1 = p2; }
        dp = Ng * (z * p1 - p0) / (z * z - 1.0);
        mu[Ng - 1 - i] = z;
        wg[Ng - 1 - i] = 2.0 / ((1.0 - z * z) * dp * dp);
    }
    for (int i = 0; i < Ng / 2; ++i) {
        double a = 0.5 * (mu[Ng - 1 - i] - mu[i]); mu[i] = -a; mu[Ng - 1 - i] = a;
        double b = 0.5 * (wg[i] + wg[Ng - 1 - i]); wg[i] = b; wg[Ng - 1 - i] = b;
    }
    if (Ng % 2) mu[Ng / 2] = 0.0;
    // SNPrep.f90:49-76: phi_j = (2j-1) pi / Nc, j outer, i inner, w = wG * 2 pi / Nc
    int ii = 0;
    for (int j = 1; j <= Nc; ++j) {
        double phi = (2 * j - 1) * PI / Nc;
        for (int i = 0; i < Ng; ++i, ++ii) {
            double st = std::sqrt(1.0 - mu[i] * mu[i]);
            k[ii * 3 + 0] = std::cos(phi) * st;
            k[ii * 3 + 1] = std::sin(phi) * st;
            k[ii * 3 + 2] = mu[i];
            w[ii] = wg[i] * (2.0 * PI / Nc);
        }
    }
    return LB_OK;
}

int lb_set_mesh(lb_handle* h, int NE, int NN, const double* rg, const int* node, const int* neighbors, const int* mat,
                int Nm) {
    if (!h) return LB_ERR_ARG;
    if (NE <= 0 || NN <= 0 || !rg || !node || !neighbors || !mat) return fail(h, LB_ERR_ARG, "lb_set_mesh: null or empty input");
    if (NE >= kMaxElems - 1) return fail(h, LB_ERR_ARG, "lb_set_mesh: at most 16777214 elements are supported");
    if (Nm < 1 || Nm > 256) return fail(h, LB_ERR_ARG, "lb_set_mesh: Nm must be in 1..256");
    if (h->device >= 0) cudaSetDevice(h->device);
    for (long long q = 0; q < 4LL * NE; ++q) {
        if (node[q] < 0 || node[q] >= NN) return fail(h, LB_ERR_ARG, "lb_set_mesh: node index out of range");
        if (neighbors[q] < -1 || neighbors[q] >= NE) return fail(h, LB_ERR_ARG, "lb_set_mesh: neighbour index out of range");
    }
    for (int e = 0; e < NE; ++e)
        if (mat[e] < 0 || mat[e] >= Nm) return fail(h, LB_ERR_ARG, "lb_set_mesh: material index out of range");
    h->NE = NE; h->NN = NN; h->Nm = Nm; h->NENK = 4LL * NE;
    h->rg.assign(rg, rg + (size_t)NN * 3);
    h->node.assign(node, node + (size_t)NE * 4);
    h->nbr.assign(neighbors, neighbors + (size_t)NE * 4);
    h->mat.assign(mat, mat + NE);
    h->nrm.assign((size_t)NE * 12, 0.0);
    h->svec.assign((size_t)NE * 12, 0.0);
    h->nbrpack.assign((size_t)NE * 4, 0u);
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(+ : bad)
    for (int e = 0; e < NE; ++e) {
        const int* nd = &h->node[(size_t)e * 4];
        double com[3] = {0, 0, 0};
        for (int q = 0; q < 4; ++q) for (int d = 0; d < 3; ++d) com[d] += h->rg[(size_t)nd[q] * 3 + d];
        for (int d = 0; d < 3; ++d) com[d] /= 4.0;
        // volume = |triple product| / 6
        double a1[3], a2[3], a3[3], cx[3];
        for (int d = 0; d < 3; ++d) {
            a1[d] = h->rg[(size_t)nd[1] * 3 + d] - h->rg[(size_t)nd[0] * 3 + d];
            a2[d] = h->rg[(size_t)nd[2] * 3 + d] - h->rg[(size_t)nd[0] * 3 + d];
            a3[d] = h->rg[(size_t)nd[3] * 3 + d] - h->rg[(size_t)nd[0] * 3 + d];
        }
        cross3(a2, a1, cx);
        double vol = std::fabs(dot3(a3, cx)) / 6.0;
        if (!(vol > 0.0)) { ++bad; continue; }
        for (int f = 0; f < 4; ++f) {
            // outward unit normal from the sorted face nodes, sign from the centroid
            // (PostProcess.f90:64-83): n = (r3-r1) x (r2-r1), r_a sorted by global id
            int fn[3] = {nd[F2K[f][0]], nd[F2K[f][1]], nd[F2K[f][2]]};
            std::sort(fn, fn + 3);
            const double* p1 = &h->rg[(size_t)fn[0] * 3];
            const double* p2 = &h->rg[(size_t)fn[1] * 3];
            const double* p3 = &h->rg[(size_t)fn[2] * 3];
            double r1[3], r2[3], n[3], c[3];
            for (int d = 0; d < 3; ++d) { r1[d] = p2[d] - p1[d]; r2[d] = p3[d] - p1[d]; c[d] = p1[d] - com[d]; }
            cross3(r2, r1, n);
            double nn = norm3(n);
            double normfac = std::copysign(1.0, dot3(n, c)) / nn;
            double area = 0.5 * nn;
            for (int d = 0; d < 3; ++d) {
                h->nrm[(size_t)e * 12 + f * 3 + d] = normfac * n[d];
                h->svec[(size_t)e * 12 + f * 3 + d] = normfac * n[d] * area / vol;
            }
            // neighbour word: element, local indices (in the neighbour) of this face's nodes
            int ep = h->nbr[(size_t)e * 4 + f];
            uint32_t word = kNoNeighbour;
            if (ep >= 0) {
                const int* ndp = &h->node[(size_t)ep * 4];
                uint32_t perm = 0;
                int found = 0;
                for (int j = 0; j < 3; ++j) {
                    int gnode = nd[F2K[f][j]];
                    for (int q = 0; q < 4; ++q) if (ndp[q] == gnode) { perm |= (uint32_t)q << (2 * j); ++found; break; }
                }
                bool back = false;
                for (int q = 0; q < 4; ++q) back |= (h->nbr[(size_t)ep * 4 + q] == e);
                if (found != 3 || !back) ++bad;
                word = (uint32_t)ep | (perm << 24);
            }
            word |= (uint32_t)((h->mat[e] >> (2 * f)) & 3) << 30;
            h->nbrpack[(size_t)e * 4 + f] = word;
        }
    }
    if (bad) return fail(h, LB_ERR_ARG, "lb_set_mesh: degenerate element or non-conforming neighbour table");
    // device geometry: per element {snx[4], sny[4], snz[4], nbrpack[4]} (64 bytes)
    std::vector<float4> geom((size_t)NE * 4);
    for (int e = 0; e < NE; ++e) {
        float4 gx, gy, gz, gw;
        float* px = &gx.x; float* py = &gy.x; float* pz = &gz.x;
        for (int f = 0; f < 4; ++f) {
            px[f] = (float)h->svec[(size_t)e * 12 + f * 3 + 0];
            py[f] = (float)h->svec[(size_t)e * 12 + f * 3 + 1];
            pz[f] = (float)h->svec[(size_t)e * 12 + f * 3 + 2];
        }
        uint32_t* pw = reinterpret_cast<uint32_t*>(&gw.x);
        for (int f = 0; f < 4; ++f) pw[f] = h->nbrpack[(size_t)e * 4 + f];
        geom[(size_t)e * 4 + 0] = gx; geom[(size_t)e * 4 + 1] = gy;
        geom[(size_t)e * 4 + 2] = gz; geom[(size_t)e * 4 + 3] = gw;
    }
    int rc = dev_upload(h, &h->d_geom, geom.data(), geom.size(), "upload geometry");
    if (rc) return rc;
    // distinct (element shape, material) types: bitwise-equal FP32 face vectors and equal material.
    // With at most 256 types every element is described by its neighbour words alone, the 8-bit type
    // index taking the place of the material bits.
    {
        constexpr int kMaxTypes = 256;
        struct Key {
            uint32_t v[13];
            bool operator==(const Key& o) const { return std::memcmp(v, o.v, sizeof v) == 0; }
        };
        struct KeyHash {
            size_t operator()(const Key& k) const {
                uint64_t x = 1469598103934665603ull;
                for (uint32_t w : k.v) x = (x ^ w) * 1099511628211ull;
                return (size_t)x;
            }
        };
        std::unordered_map<Key, int, KeyHash> types;
        std::vector<int> idx(NE);
        std::vector<float4> tab;
        std::vector<int> tmat;
        bool ok = true;
        for (int e = 0; e < NE && ok; ++e) {
            Key k;
            std::memcpy(k.v, &geom[(size_t)e * 4], 48);
            k.v[12] = (uint32_t)h->mat[e];
            auto it = types.find(k);
            if (it == types.end()) {
                if ((int)types.size() >= kMaxTypes) { ok = false; break; }
                it = types.emplace(k, (int)types.size()).first;
                tab.push_back(geom[(size_t)e * 4 + 0]);
                tab.push_back(geom[(size_t)e * 4 + 1]);
                tab.push_back(geom[(size_t)e * 4 + 2]);
                tmat.push_back(h->mat[e]);
            }
            idx[e] = it->second;
        }
        h->ngeom = 0;
        if (ok) {
            std::vector<int4> rec(NE);
            for (int e = 0; e < NE; ++e) {
                uint32_t w[4];
                for (int f = 0; f < 4; ++f)
                    w[f] = (h->nbrpack[(size_t)e * 4 + f] & 0x3FFFFFFFu) | ((uint32_t)((idx[e] >> (2 * f)) & 3) << 30);
                rec[e] = make_int4((int)w[0], (int)w[1], (int)w[2], (int)w[3]);
            }
            if ((rc = dev_upload(h, &h->d_rec, rec.data(), rec.size(), "upload element records"))) return rc;
            if ((rc = dev_upload(h, &h->d_gtab, tab.data(), tab.size(), "upload type table"))) return rc;
            if ((rc = dev_upload(h, &h->d_tmat, tmat.data(), tmat.size(), "upload type materials"))) return rc;
            h->ngeom = (int)types.size();
        }
    }
    rc = dev_upload(h, &h->d_mat, h->mat.data(), h->mat.size(), "upload materials");
    if (rc) return rc;
    h->mesh_ready = true;
    ++h->mesh_version;
    h->angle_ready = false;
    h->phys_ready = false;
    return LB_OK;
}

// Cluster schedule (sweep_cluster_kernel): blocks of kClusterSize consecutive elements (a hex of a
// box mesh split into 6 tets is one block) are swept as units, one thread per block taking its
// elements in level order, so a block's sources and solutions (96 contiguous bytes) are read and
// written together.  Per direction the block graph (block B depends on block A when an element of B
// has an upstream neighbour in A) must be acyclic; its longest-path levels order the blocks, and
// blocks with the same element order and face masks are adjacent inside a level.  Record of a block:
//   x: block index;  y, z, w: two 16-bit slots each, in execution order: element offset in the
//   block (3 b, 7 = empty) | upstream-face mask << 3 | outflow-face mask << 7.
// Built on device handles; when some direction's block graph has a cycle no cluster schedule is
// kept and the sweep uses the element schedules.
// Blocks of the cluster schedule.  Box meshes number the 6 tets of a hex consecutively, so blocks of
// kClusterSize consecutive ids are face-connected and need no member table (blk_elem stays empty).
// Other meshes get blocks grown greedily: elements are visited in Morton order of their centroids, and
// a block grows from its first element by the unassigned face neighbour sharing the most faces with
// the block's members (then the earliest in Morton order), up to kClusterSize elements.
static void form_blocks(Handle* h, std::vector<int>& blk_elem, std::vector<int>& blk_of, std::vector<int>& blk_pos) {
    constexpr int K = kClusterSize;
    const int NE = h->NE;
    blk_elem.clear();
    blk_of.assign(NE, 0);
    blk_pos.assign(NE, 0);
    bool consecutive = true;
    for (int b0 = 0; b0 < NE && consecutive; b0 += K) {
        const int n = std::min(K, NE - b0);
        // face-connected: a flood fill from the first member reaches all n
        int reached = 1, mask = 1;
        for (bool grew = true; grew;) {
            grew = false;
            for (int q = 0; q < n; ++q) {
                if (!((mask >> q) & 1)) continue;
                for (int f = 0; f < 4; ++f) {
                    const int ep = h->nbr[(size_t)(b0 + q) * 4 + f] - b0;
                    if (ep >= 0 && ep < n && !((mask >> ep) & 1)) { mask |= 1 << ep; ++reached; grew = true; }
                }
            }
        }
        consecutive = reached == n;
    }
    if (consecutive) {
        for (int e = 0; e < NE; ++e) { blk_of[e] = e / K; blk_pos[e] = e % K; }
        return;
    }
    // Morton order of the centroids (21 bits per axis)
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int v = 0; v < h->NN; ++v)
        for (int d = 0; d < 3; ++d) {
            lo[d] = std::min(lo[d], h->rg[(size_t)v * 3 + d]);
            hi[d] = std::max(hi[d], h->rg[(size_t)v * 3 + d]);
        }
    auto spread = [](uint64_t x) {
        x &= 0x1FFFFF;
        x = (x | x << 32) & 0x1F00000000FFFFull;
        x = (x | x << 16) & 0x1F0000FF0000FFull;
        x = (x | x << 8) & 0x100F00F00F00F00Full;
        x = (x | x << 4) & 0x10C30C30C30C30C3ull;
        x = (x | x << 2) & 0x1249249249249249ull;
        return x;
    };
    std::vector<std::pair<uint64_t, int>> key(NE);
    for (int e = 0; e < NE; ++e) {
        uint64_t code = 0;
        for (int d = 0; d < 3; ++d) {
            double c = 0.0;
            for (int k = 0; k < 4; ++k) c += h->rg[(size_t)h->node[(size_t)e * 4 + k] * 3 + d];
            const double t = (0.25 * c - lo[d]) / std::max(hi[d] - lo[d], 1e-300);
            code |= spread((uint64_t)std::min(2097151.0, std::max(0.0, t * 2097151.0))) << d;
        }
        key[e] = {code, e};
    }
    std::sort(key.begin(), key.end());
    std::vector<int> rank(NE);
    for (int q = 0; q < NE; ++q) rank[key[q].second] = q;
    std::vector<int> owner(NE, -1), members;
    int nb = 0;
    for (int q = 0; q < NE; ++q) {
        const int seed = key[q].second;
        if (owner[seed] >= 0) continue;
        members.assign(1, seed);
        owner[seed] = nb;
        while ((int)members.size() < K) {
            int best = -1, best_shared = 0;
            for (int m : members)
                for (int f = 0; f < 4; ++f) {
                    const int c = h->nbr[(size_t)m * 4 + f];
                    if (c < 0 || owner[c] >= 0) continue;
                    int shared = 0;
                    for (int g = 0; g < 4; ++g) {
                        const int cn = h->nbr[(size_t)c * 4 + g];
                        shared += cn >= 0 && owner[cn] == nb;
                    }
                    if (best < 0 || shared > best_shared || (shared == best_shared && rank[c] < rank[best])) {
                        best = c;
                        best_shared = shared;
                    }
                }
            if (best < 0) break;
            owner[best] = nb;
            members.push_back(best);
        }
        for (int k = 0; k < K; ++k) blk_elem.push_back(k < (int)members.size() ? members[k] : -1);
        for (int k = 0; k < (int)members.size(); ++k) { blk_of[members[k]] = nb; blk_pos[members[k]] = k; }
        ++nb;
    }
}

// Units per group of the block schedule: the sweep's CTA size (512 threads), LB_CLUSTER_GROUP=<n> for
// another cap, 0 for uncapped groups (Kahn's levels).
static int cluster_group_cap() {
    const char* e = std::getenv("LB_CLUSTER_GROUP");
    if (e && *e) return std::max(0, std::atoi(e));
    return 512;
}

// Block schedule of every direction: units in groups (a group's units depend only on units of earlier
// groups; the sweep runs a group between two CTA barriers).  A unit is a block, or part of one: Kahn's
// algorithm runs over the units of the direction, and whenever no unit is ready while elements remain
// (the direction's block graph has a cycle), every element whose upstream neighbours are all done
// leaves its unit for a new unit with the other such elements of its block.  Those elements are
// mutually independent, so the new unit is valid and ready, and the sweep always progresses.  A record
// per unit: the block index, then up to kClusterSize 16-bit slots in execution order (position in the
// block, upstream-face mask << 3, outflow-face mask << 7; position 7 = empty slot), the unit's elements
// ordered by element level.
static int build_cluster_schedule(Handle* h) {
    constexpr int K = kClusterSize;
    h->nclusters = 0;
    h->max_cluster_levels = 0;
    h->max_cluster_records = 0;
    h->cl_start_h.clear();
    h->crec_h.clear();
    h->cl_base_h.clear();
    h->ncl_h.clear();
    h->crec_base_h.clear();
    h->blk_elem_h.clear();
    for (void** p : {(void**)&h->d_crec, (void**)&h->d_cl_start, (void**)&h->d_cl_base, (void**)&h->d_ncl,
                     (void**)&h->d_crec_base, (void**)&h->d_blk_elem})
        if (*p) {
            cudaFree(*p);
            *p = nullptr;
        }
    const int NE = h->NE, NI = h->NI;
    if (NE < K) return LB_OK;
    std::vector<int> blk_elem, blk_of, blk_pos;
    form_blocks(h, blk_elem, blk_of, blk_pos);
    const int NC = blk_elem.empty() ? (NE + K - 1) / K : (int)(blk_elem.size() / K);
    std::vector<std::vector<int4>> crec(NI);
    std::vector<std::vector<int>> cstart(NI);
    bool cyclic = false;
    // Units per group.  A group is one pass of the sweep CTA's threads between two barriers, so a group of
    // Kahn's levels (all ready units) with more units than threads takes several passes, the last one part
    // empty; capped groups pack every pass (list scheduling: ready units wait at most until a pass has room).
    const int cap = cluster_group_cap();
#pragma omp parallel reduction(|| : cyclic)
    {
        std::vector<int> lev(NE), unit(NE), ublk, pend, epend, dstart(NE + 1), ddst, cur, nxt, members, ord, waiting;
        std::vector<int> usize, newunit, rest;
        std::vector<char> done(NE);
        std::vector<uint16_t> fld(NE);
        std::vector<unsigned long long> key;
        std::vector<int4> tmp;
        std::vector<std::vector<int>> umem;
        // Walk order inside a block: of the orders that respect the block's internal dependencies, the one
        // with the fewest upstream neighbours three or more updates back (the kernel holds the last two
        // solutions in registers; earlier ones are read back through L1), ties broken towards the
        // (element level, id) order.  The best order depends only on the block's dependency pattern
        // (which member reads which), so it is memoised by that pattern.
        std::unordered_map<unsigned long long, unsigned> best_order;
        auto order_block = [&](std::vector<int>& mem, int c) {
            const int nmem = (int)mem.size();
            if (nmem <= 3) return;   // with three or fewer updates every upstream read is within two
            int upmask[kClusterSize] = {0, 0, 0, 0, 0, 0};
            unsigned long long sig = (unsigned long long)nmem;
            for (int a = 0; a < nmem; ++a) {
                const int x = mem[a];
                const int upm = (fld[x] >> 3) & 0xF;
                for (int f = 0; f < 4; ++f) {
                    if (!((upm >> f) & 1)) continue;
                    const int y = h->nbr[(size_t)x * 4 + f];
                    if (y < 0 || unit[y] != c) continue;
                    for (int b = 0; b < nmem; ++b)
                        if (mem[b] == y) upmask[a] |= 1 << b;
                }
                sig |= (unsigned long long)upmask[a] << (4 + 6 * a);
            }
            unsigned code;
            auto hit = best_order.find(sig);
            if (hit != best_order.end()) {
                code = hit->second;
            } else {
                // depth-first over the orders that respect the dependencies, members tried in their sorted order
                int perm[kClusterSize], pos[kClusterSize], bperm[kClusterSize];
                int bcost = 1 << 30;
                for (int a = 0; a < nmem; ++a) pos[a] = -1;
                std::function<void(int, int, int)> dfs = [&](int depth, int used, int cost) {
                    if (cost >= bcost) return;
                    if (depth == nmem) {
                        bcost = cost;
                        std::copy(perm, perm + nmem, bperm);
                        return;
                    }
                    for (int a = 0; a < nmem; ++a) {
                        if ((used >> a) & 1) continue;
                        if ((upmask[a] & used) != upmask[a]) continue;
                        int far = 0;
                        for (int b = 0; b < nmem; ++b)
                            if (((upmask[a] >> b) & 1) && depth - pos[b] > 2) ++far;
                        perm[depth] = a;
                        pos[a] = depth;
                        dfs(depth + 1, used | (1 << a), cost + far);
                        pos[a] = -1;
                    }
                };
                dfs(0, 0, 0);
                code = 0;
                for (int k = 0; k < nmem; ++k) code |= (unsigned)bperm[k] << (3 * k);
                best_order.emplace(sig, code);
            }
            int tmpm[kClusterSize];
            for (int k = 0; k < nmem; ++k) tmpm[k] = mem[(code >> (3 * k)) & 7];
            for (int k = 0; k < nmem; ++k) mem[k] = tmpm[k];
        };
#pragma omp for schedule(dynamic, 1)
        for (int i = 0; i < NI; ++i) {
            if (cyclic) continue;
            const int* it = &h->items[(size_t)i * NE];
            const int* st = &h->lvl_start[h->lvl_base[i]];
            for (int L = 0; L < h->nlev[i]; ++L)
                for (int es = st[L]; es < st[L + 1]; ++es) lev[it[es] & 0xFFFFFF] = L;
            for (int es = 0; es < NE; ++es) {
                const int e = it[es] & 0xFFFFFF;
                fld[e] = (uint16_t)(blk_pos[e] | (((it[es] >> 24) & 0xF) << 3) | (((it[es] >> 28) & 0xF) << 7));
            }
            // element edges y -> x (y upstream of x), as downstream lists
            std::fill(dstart.begin(), dstart.end(), 0);
            epend.assign(NE, 0);
            for (int x = 0; x < NE; ++x) {
                const int upm = (fld[x] >> 3) & 0xF;
                for (int f = 0; f < 4; ++f)
                    if ((upm >> f) & 1) { ++dstart[h->nbr[(size_t)x * 4 + f] + 1]; ++epend[x]; }
            }
            for (int e = 0; e < NE; ++e) dstart[e + 1] += dstart[e];
            ddst.resize(dstart[NE]);
            {
                std::vector<int> fill(dstart.begin(), dstart.end() - 1);
                for (int x = 0; x < NE; ++x) {
                    const int upm = (fld[x] >> 3) & 0xF;
                    for (int f = 0; f < 4; ++f)
                        if ((upm >> f) & 1) ddst[fill[h->nbr[(size_t)x * 4 + f]]++] = x;
                }
            }
            // units start as the blocks; pend[u] = edges into u from elements of other, unfinished units
            ublk.resize(NC);
            umem.assign(NC, {});
            for (int c = 0; c < NC; ++c) ublk[c] = c;
            for (int e = 0; e < NE; ++e) { unit[e] = blk_of[e]; umem[unit[e]].push_back(e); done[e] = 0; }
            pend.assign(NC, 0);
            for (int y = 0; y < NE; ++y)
                for (int j = dstart[y]; j < dstart[y + 1]; ++j)
                    if (unit[ddst[j]] != unit[y]) ++pend[unit[ddst[j]]];
            cur.clear();
            waiting.clear();
            for (int c = 0; c < NC; ++c)
                if (pend[c] == 0 && !umem[c].empty()) cur.push_back(c);
            for (int e = 0; e < NE; ++e)
                if (epend[e] == 0 && pend[unit[e]] > 0) waiting.push_back(e);
            std::vector<int4>& out = crec[i];
            out.clear();
            cstart[i].clear();
            int ndone = 0;
            while (ndone < NE) {
                // at most `cap` units per group (one per thread of the sweep CTA): the ready units past it wait
                // for the next group, ahead of the units that become ready now
                rest.clear();
                if (cap > 0 && (int)cur.size() > cap) {
                    // the units ready longest go first (the leftovers of the previous group lead `cur`)
                    rest.assign(cur.begin() + cap, cur.end());
                    cur.resize(cap);
                }
                if (cur.empty()) {
                    // stalled on a cycle of units: the ready elements of every blocked unit form new units
                    newunit.clear();
                    std::sort(waiting.begin(), waiting.end(), [&](int x, int y) { return unit[x] < unit[y]; });
                    for (size_t q = 0; q < waiting.size();) {
                        const int u = unit[waiting[q]];
                        size_t r = q;
                        while (r < waiting.size() && unit[waiting[r]] == u) ++r;
                        const int nu = (int)umem.size();
                        umem.emplace_back(waiting.begin() + q, waiting.begin() + r);
                        ublk.push_back(ublk[u]);
                        pend.push_back(0);
                        for (size_t t = q; t < r; ++t) unit[waiting[t]] = nu;
                        std::vector<int>& m0 = umem[u];
                        m0.erase(std::remove_if(m0.begin(), m0.end(), [&](int x) { return unit[x] == nu; }), m0.end());
                        // edges from the moved elements to the rest of their old unit now cross units
                        for (size_t t = q; t < r; ++t)
                            for (int j = dstart[waiting[t]]; j < dstart[waiting[t] + 1]; ++j)
                                if (unit[ddst[j]] == u) ++pend[u];
                        newunit.push_back(nu);
                        q = r;
                    }
                    waiting.clear();
                    if (newunit.empty()) break;   // an element-level cycle: no block schedule
                    cur.swap(newunit);
                }
                cstart[i].push_back((int)out.size());
                const int n = (int)cur.size();
                tmp.resize(n);
                key.resize(n);
                for (int q = 0; q < n; ++q) {
                    const int c = cur[q];
                    members = umem[c];
                    std::sort(members.begin(), members.end(),
                              [&](int x, int y) { return lev[x] != lev[y] ? lev[x] < lev[y] : x < y; });
                    order_block(members, c);
                    uint32_t sl[6];
                    for (int k = 0; k < 6; ++k) sl[k] = k < (int)members.size() ? fld[members[k]] : 7u;
                    tmp[q] = make_int4(ublk[c], (int)(sl[0] | (sl[1] << 16)), (int)(sl[2] | (sl[3] << 16)),
                                       (int)(sl[4] | (sl[5] << 16)));
                    key[q] = ((unsigned long long)(uint32_t)tmp[q].y * 0x9E3779B97F4A7C15ull) ^
                             ((unsigned long long)(uint32_t)tmp[q].z << 21) ^ (uint32_t)tmp[q].w;
                }
                // units with equal patterns next to each other (a warp then runs one element sequence), and
                // among them by block index, so that a warp's blocks lie close together in memory
                ord.resize(n);
                for (int q = 0; q < n; ++q) ord[q] = q;
                std::sort(ord.begin(), ord.end(), [&](int x, int y) {
                    return key[x] != key[y] ? key[x] < key[y] : tmp[x].x != tmp[y].x ? tmp[x].x < tmp[y].x : x < y;
                });
                for (int q = 0; q < n; ++q) out.push_back(tmp[ord[q]]);
                nxt.clear();
                for (int c : cur)
                    for (int y : umem[c]) {
                        done[y] = 1;
                        ++ndone;
                    }
                for (int c : cur)
                    for (int y : umem[c])
                        for (int j = dstart[y]; j < dstart[y + 1]; ++j) {
                            const int x = ddst[j];
                            const int ux = unit[x];
                            if (ux != c && --pend[ux] == 0) nxt.push_back(ux);
                            if (--epend[x] == 0 && !done[x]) waiting.push_back(x);
                        }
                // elements whose units became ready do not wait
                waiting.erase(std::remove_if(waiting.begin(), waiting.end(), [&](int x) { return pend[unit[x]] == 0; }),
                              waiting.end());
                rest.insert(rest.end(), nxt.begin(), nxt.end());
                cur.swap(rest);
            }
            cstart[i].push_back((int)out.size());
            if (ndone != NE) cyclic = true;   // an element-level cycle: no block schedule
        }
    }
    if (cyclic) return LB_OK;
    std::vector<int> cl_start, cl_base(NI), ncl(NI);
    std::vector<long long> base(NI + 1, 0);
    int maxl = 0, maxr = 0;
    for (int i = 0; i < NI; ++i) {
        cl_base[i] = (int)cl_start.size();
        ncl[i] = (int)cstart[i].size() - 1;
        maxl = std::max(maxl, ncl[i]);
        maxr = std::max(maxr, (int)crec[i].size());
        cl_start.insert(cl_start.end(), cstart[i].begin(), cstart[i].end());
        base[i + 1] = base[i] + (long long)crec[i].size();
    }
    std::vector<int4> all((size_t)base[NI]);
    for (int i = 0; i < NI; ++i) std::copy(crec[i].begin(), crec[i].end(), all.begin() + base[i]);
    crec.clear();
    int rc = dev_upload(h, &h->d_crec, all.data(), all.size(), "upload cluster records");
    if (!rc) rc = dev_upload(h, &h->d_crec_base, base.data(), base.size(), "upload cluster record offsets");
    if (!rc && !blk_elem.empty()) rc = dev_upload(h, &h->d_blk_elem, blk_elem.data(), blk_elem.size(), "upload blocks");
    if (!rc) rc = dev_upload(h, &h->d_cl_start, cl_start.data(), cl_start.size(), "upload cluster levels");
    if (!rc) rc = dev_upload(h, &h->d_cl_base, cl_base.data(), cl_base.size(), "upload cluster level offsets");
    if (!rc) rc = dev_upload(h, &h->d_ncl, ncl.data(), ncl.size(), "upload cluster level counts");
    if (rc) return rc;
    h->nclusters = NC;
    h->max_cluster_levels = maxl;
    h->max_cluster_records = maxr;
    h->cluster_levels_total = 0;
    for (int i = 0; i < NI; ++i) h->cluster_levels_total += ncl[i];
    h->cl_start_h = cl_start;
    h->cl_base_h = cl_base;
    h->crec_base_h = base;
    h->blk_elem_h = blk_elem;
    if (h->device < 0) h->crec_h = std::move(all);   // host-only handles keep the records for queries
    h->ncl_h = ncl;
    return LB_OK;
}

int lb_set_quadrature(lb_handle* h, int NI, const double* k, const double* w) {
    if (!h) return LB_ERR_ARG;
    if (!h->mesh_ready) return fail(h, LB_ERR_STATE, "lb_set_quadrature: mesh not set");
    if (NI <= 0 || NI >= (1 << 24) || !k || !w) return fail(h, LB_ERR_ARG, "lb_set_quadrature: bad NI or null input");
    if (h->device >= 0) cudaSetDevice(h->device);
    const int NE = h->NE;
    h->NI = NI;
    h->NIpad = (NI + 15) / 16 * 16;
    h->k.assign(k, k + (size_t)NI * 3);
    h->w.assign(w, w + NI);
    h->items.assign((size_t)NI * NE, 0);
    std::vector<std::vector<int>> starts(NI);
    std::vector<long long> nz(NI, 0);
    int cyc = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : cyc)
    for (int i = 0; i < NI; ++i)
        if (!build_direction(h, i, &h->items[(size_t)i * NE], starts[i], nz[i])) ++cyc;
    if (cyc) {
        h->angle_ready = false;
        return fail(h, LB_ERR_CYCLE, "SweepOrder: Sweep is stagnant. Check the mesh for errors, as this may imply "
                                     "discontinuity in face/element indexing.");
    }
    h->nlev.assign(NI, 0);
    h->lvl_base.assign(NI + 1, 0);
    h->lvl_start.clear();
    h->nz_upstream = 0;
    int maxlev = 0;
    for (int i = 0; i < NI; ++i) {
        h->nlev[i] = (int)starts[i].size() - 1;
        h->lvl_base[i] = (int)h->lvl_start.size();
        h->lvl_start.insert(h->lvl_start.end(), starts[i].begin(), starts[i].end());
        h->nz_upstream += nz[i];
        maxlev = std::max(maxlev, h->nlev[i]);
    }
    h->lvl_base[NI] = (int)h->lvl_start.size();
    // global level ids: gid(i, L) = sum_{i'<i} nlev[i'] + L
    std::vector<int> gbase(NI + 1, 0);
    for (int i = 0; i < NI; ++i) gbase[i + 1] = gbase[i] + h->nlev[i];
    h->total_levels = gbase[NI];
    // chunk list, level-major across directions: every chunk's dependencies (the previous level
    // of its own direction) precede it, so claiming chunks in order can never deadlock.
    std::vector<int4> chunks;
    chunks.reserve((size_t)NI * NE / 24 + 16);
    for (int L = 0; L < maxlev; ++L)
        for (int i = 0; i < NI; ++i) {
            if (L >= h->nlev[i]) continue;
            const int* st = &h->lvl_start[h->lvl_base[i]];
            int a = st[L], b = st[L + 1];
            int prev = (L > 0) ? (st[L] - st[L - 1]) : 0;
            for (int s = a; s < b; s += 32) {
                int n = std::min(32, b - s);
                chunks.push_back(make_int4(i | ((n - 1) << 24), s, gbase[i] + L, prev));
            }
        }
    if (chunks.size() >= (size_t)INT32_MAX) return fail(h, LB_ERR_ARG, "lb_set_quadrature: problem too large");
    h->nchunks = (int)chunks.size();
    // Execution order on the device: inside every level the elements are grouped by upstream-face
    // mask (ascending element id within a group).  Elements of a level are independent, so the
    // results do not change, but a warp then runs the face bodies of about 2 upstream faces instead
    // of the union of its elements' masks (3.7 of 4 at config1).  lb_get_schedule keeps returning
    // the reference's order (h->items).
    std::vector<int> exec_items(h->device >= 0 ? h->items.size() : 0);
#pragma omp parallel for schedule(dynamic, 4)
    for (int i = 0; i < (h->device >= 0 ? NI : 0); ++i) {
        const int* src = h->items.data() + (size_t)i * NE;
        int* dst = exec_items.data() + (size_t)i * NE;
        for (int L = 0; L < h->nlev[i]; ++L) {
            const int a = h->lvl_start[h->lvl_base[i] + L], b = h->lvl_start[h->lvl_base[i] + L + 1];
            int cnt[17] = {0};
            for (int es = a; es < b; ++es) ++cnt[((src[es] >> 24) & 0xF) + 1];
            for (int k = 1; k < 17; ++k) cnt[k] += cnt[k - 1];
            for (int es = a; es < b; ++es) dst[a + cnt[(src[es] >> 24) & 0xF]++] = src[es];
        }
    }
    int rc = dev_upload(h, &h->d_items, exec_items.data(), exec_items.size(), "upload sweep items");
    if (rc) return rc;
    rc = build_cluster_schedule(h);
    if (rc) return rc;
    rc = dev_upload(h, &h->d_chunks, chunks.data(), chunks.size(), "upload sweep chunks");
    if (rc) return rc;
    rc = dev_alloc(h, &h->d_done, (size_t)h->total_levels, "level counters");
    if (rc) return rc;
    {
        // items with every level padded to a multiple of 32 (padding = -1): a 32-element chunk of the
        // padded order never spans two levels, so its elements never depend on each other
        std::vector<long long> pbase(NI + 1, 0);
        for (int i = 0; i < NI; ++i) {
            long long len = 0;
            const int* st = &h->lvl_start[h->lvl_base[i]];
            for (int L = 0; L < h->nlev[i]; ++L) len += ((st[L + 1] - st[L]) + 31) / 32 * 32;
            pbase[i + 1] = pbase[i] + len;
        }
        std::vector<int> pitems((size_t)pbase[NI], -1);
#pragma omp parallel for schedule(dynamic, 4)
        for (int i = 0; i < NI; ++i) {
            const int* st = &h->lvl_start[h->lvl_base[i]];
            long long o = pbase[i];
            for (int L = 0; L < h->nlev[i]; ++L) {
                for (int es = st[L]; es < st[L + 1]; ++es) pitems[(size_t)o++] = h->items[(size_t)i * NE + es];
                o = pbase[i] + (o - pbase[i] + 31) / 32 * 32;
            }
        }
        h->npitems = pbase[NI];
        rc = dev_upload(h, &h->d_pitems, pitems.data(), pitems.size(), "upload padded items");
        if (rc) return rc;
        rc = dev_upload(h, &h->d_pbase, pbase.data(), pbase.size(), "upload padded offsets");
        if (rc) return rc;
    }
    rc = dev_upload(h, &h->d_lvl_start, h->lvl_start.data(), h->lvl_start.size(), "upload level starts");
    if (rc) return rc;
    rc = dev_upload(h, &h->d_lvl_base, h->lvl_base.data(), h->lvl_base.size(), "upload level offsets");
    if (rc) return rc;
    rc = dev_upload(h, &h->d_nlev, h->nlev.data(), h->nlev.size(), "upload level counts");
    if (rc) return rc;
    {
        // classes of directions with identical schedules (exact comparison after a hash)
        std::vector<unsigned long long> hsh(NI);
#pragma omp parallel for schedule(static)
        for (int i = 0; i < NI; ++i) {
            unsigned long long x = 1469598103934665603ULL ^ (unsigned long long)h->nlev[i];
            const int* it = &h->items[(size_t)i * NE];
            for (int es = 0; es < NE; ++es) { x ^= (unsigned)it[es]; x *= 1099511628211ULL; }
            hsh[i] = x;
        }
        h->dir_class.assign(NI, -1);
        for (int i = 0; i < NI; ++i) {
            if (h->dir_class[i] >= 0) continue;
            h->dir_class[i] = i;
            for (int j = i + 1; j < NI; ++j) {
                if (h->dir_class[j] >= 0 || hsh[j] != hsh[i] || h->nlev[j] != h->nlev[i]) continue;
                if (std::memcmp(&h->items[(size_t)i * NE], &h->items[(size_t)j * NE], sizeof(int) * (size_t)NE) == 0 &&
                    std::equal(&h->lvl_start[h->lvl_base[i]], &h->lvl_start[h->lvl_base[i]] + h->nlev[i] + 1,
                               &h->lvl_start[h->lvl_base[j]]))
                    h->dir_class[j] = i;
            }
        }
        h->class_members.clear();
        h->class_start.assign(1, 0);
        for (int i = 0; i < NI; ++i) {
            if (h->dir_class[i] != i) continue;
            for (int j = i; j < NI; ++j)
                if (h->dir_class[j] == i) h->class_members.push_back(j);
            h->class_start.push_back((int)h->class_members.size());
        }
        h->groups_gmax = 0;
        h->ngroups = 0;
    }
    h->sweep_cfg = -1;
    h->sweep_trial = 0;
    h->sweep_trial_ms.clear();
    h->sweep_finalists.clear();
    std::vector<float4> dirs(NI);
    for (int i = 0; i < NI; ++i)
        dirs[i] = make_float4((float)k[i * 3], (float)k[i * 3 + 1], (float)k[i * 3 + 2], (float)w[i]);
    rc = dev_upload(h, &h->d_dirs, dirs.data(), dirs.size(), "upload directions");
    if (rc) return rc;
    size_t pe = (size_t)NI * (size_t)h->NENK;
    if (h->device >= 0 && h->psi_elems != pe) {
        rc = dev_alloc(h, &h->d_psi, pe, "angular work vector");
        if (rc) return rc;
        if (h->d_qext) { cudaFree(h->d_qext); h->d_qext = nullptr; }
        h->psi_elems = pe;
    }
    h->angle_ready = true;
    h->phys_ready = false;
    return LB_OK;
}

int lb_get_schedule(lb_handle* h, int* sl, unsigned char* upmask, int* nlevels, int* level_start) {
    if (!h) return LB_ERR_ARG;
    if (!h->angle_ready) return fail(h, LB_ERR_STATE, "lb_get_schedule: quadrature not set");
    const int NE = h->NE, NI = h->NI;
    for (size_t q = 0; q < (size_t)NI * NE; ++q) {
        int it = h->items[q];
        if (sl) sl[q] = it & (kMaxElems - 1);
        if (upmask) upmask[q] = (unsigned char)((it >> 24) & 0xF);
    }
    for (int i = 0; i < NI; ++i) {
        if (nlevels) nlevels[i] = h->nlev[i];
        if (level_start)
            for (int L = 0; L <= h->nlev[i]; ++L) level_start[(size_t)i * (NE + 1) + L] = h->lvl_start[h->lvl_base[i] + L];
    }
    return LB_OK;
}

int lb_set_xs(lb_handle* h, int Ls, const double* sigt, const double* sigs) {
    if (!h) return LB_ERR_ARG;
    if (!h->angle_ready) return fail(h, LB_ERR_STATE, "lb_set_xs: quadrature not set");
    if (Ls < 0 || Ls > 15 || !sigt || !sigs) return fail(h, LB_ERR_ARG, "lb_set_xs: Ls must be in 0..15");
    if (h->device >= 0) cudaSetDevice(h->device);
    const int Nm = h->Nm, NI = h->NI, NIpad = h->NIpad;
    for (int m = 0; m < Nm; ++m)
        if (!(sigt[m] >= 0.0) || !std::isfinite(sigt[m])) return fail(h, LB_ERR_NAN, "lb_set_xs: invalid total cross section");
    h->sigt.assign(sigt, sigt + Nm);
    h->sigs.assign(sigs, sigs + (size_t)Nm * (Ls + 1));
    ++h->xs_version;
    int nm = (Ls + 1) * (Ls + 1);
    int nmpad = (nm + 15) / 16 * 16;
    bool rebuild = (Ls != h->Ls) || (h->ybuilt_NI != NI);
    h->Ls = Ls; h->nm = nm; h->nmpad = nmpad;
    int rc;
    std::vector<float> st(Nm);
    for (int m = 0; m < Nm; ++m) st[m] = (float)sigt[m];
    rc = dev_upload(h, &h->d_sigt, st.data(), st.size(), "upload sigt");
    if (rc) return rc;
    std::vector<float> sl((size_t)Nm * nmpad, 0.f);
    for (int m = 0; m < Nm; ++m)
        for (int l = 0; l <= Ls; ++l)
            for (int j = l * l; j < (l + 1) * (l + 1); ++j) sl[(size_t)m * nmpad + j] = (float)sigs[(size_t)m * (Ls + 1) + l];
    rc = dev_upload(h, &h->d_sigl, sl.data(), sl.size(), "upload sigma_l");
    if (rc) return rc;
    if (rebuild || !h->d_Ym2d) {
        // split Y into three BF16 planes (hi + mid + lo carries 24 significant bits)
        std::vector<__nv_bfloat16> ym((size_t)3 * NIpad * nmpad), yd((size_t)3 * nmpad * NIpad);
        std::vector<double> Y(nm);
        auto split3 = [](double v, __nv_bfloat16* o3) {
            float f = (float)v;
            __nv_bfloat16 a = __float2bfloat16_rn(f);
            float r1 = f - __bfloat162float(a);
            __nv_bfloat16 b = __float2bfloat16_rn(r1);
            float r2 = r1 - __bfloat162float(b);
            o3[0] = a; o3[1] = b; o3[2] = __float2bfloat16_rn(r2);
        };
        for (auto& v : ym) v = __float2bfloat16_rn(0.f);
        for (auto& v : yd) v = __float2bfloat16_rn(0.f);
        for (int i = 0; i < NI; ++i) {
            real_sh(Ls, &h->k[(size_t)i * 3], Y.data());
            for (int j = 0; j < nm; ++j) {
                __nv_bfloat16 o3[3];
                split3(Y[j], o3);
                for (int p = 0; p < 3; ++p) ym[((size_t)p * NIpad + i) * nmpad + j] = o3[p];
                split3(h->w[i] * Y[j], o3);
                for (int p = 0; p < 3; ++p) yd[((size_t)p * nmpad + j) * NIpad + i] = o3[p];
            }
        }
        rc = dev_upload(h, &h->d_Ym2d, ym.data(), ym.size(), "upload M2D operator");
        if (rc) return rc;
        rc = dev_upload(h, &h->d_Yd2m, yd.data(), yd.size(), "upload D2M operator");
        if (rc) return rc;
        h->ybuilt_NI = NI;
    }
    h->phys_ready = true;
    return LB_OK;
}

int lb_get_timers(lb_handle* h, double* ms, long long* launches) {
    if (!h) return LB_ERR_ARG;
    if (h->device < 0) return fail(h, LB_ERR_STATE, "host-only handle");
    cudaSetDevice(h->device);
    timers_flush(h);
    for (int q = 0; q < LB_NTIMERS; ++q) {
        if (ms) ms[q] = h->acc_ms[q];
        if (launches) launches[q] = h->launches[q];
    }
    return LB_OK;
}

int lb_reset_timers(lb_handle* h) {
    if (!h) return LB_ERR_ARG;
    if (h->device < 0) return fail(h, LB_ERR_STATE, "host-only handle");
    cudaSetDevice(h->device);
    timers_flush(h);
    for (int q = 0; q < LB_NTIMERS; ++q) { h->acc_ms[q] = 0; h->launches[q] = 0; }
    return LB_OK;
}

int lb_sweep_stats(lb_handle* h, double* bytes, double* updates, long long* upfaces) {
    if (!h || !h->angle_ready) return LB_ERR_STATE;
    double upd = (double)h->NE * h->NI;
    // algorithmic bytes of one sweep: per update the FP32 source read (16 B) and solution write
    // (16 B), 3 FP32 face-node values per upstream face (12 B), and the compact element record once
    // per sweep (16 B with the type table, 64 B without).  Schedule records are not counted.
    double b = upd * (16.0 + 16.0) + 12.0 * (double)h->nz_upstream + (h->ngeom ? 16.0 : 64.0) * h->NE;
    if (bytes) *bytes = b;
    if (updates) *updates = upd;
    if (upfaces) *upfaces = h->nz_upstream;
    return LB_OK;
}

int lb_mark(lb_handle* h, int slot) {
    if (!h || slot < 0 || slot >= 16) return LB_ERR_ARG;
    if (h->device < 0) return fail(h, LB_ERR_STATE, "host-only handle");
    cudaSetDevice(h->device);
    if (!h->marks[slot] && cudaEventCreate(&h->marks[slot]) != cudaSuccess) return fail(h, LB_ERR_CUDA, "event create");
    cudaError_t e = cudaEventRecord(h->marks[slot], h->stream);
    return e == cudaSuccess ? LB_OK : cuda_fail(h, e, "event record");
}

int lb_elapsed_ms(lb_handle* h, int a, int b, double* ms) {
    if (!h || !ms || a < 0 || b < 0 || a >= 16 || b >= 16 || !h->marks[a] || !h->marks[b]) return LB_ERR_ARG;
    cudaSetDevice(h->device);
    cudaError_t e = cudaEventSynchronize(h->marks[b]);
    float f = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&f, h->marks[a], h->marks[b]);
    if (e != cudaSuccess) return cuda_fail(h, e, "event elapsed");
    *ms = f;
    return LB_OK;
}

int lb_get_sweep_config(lb_handle* h, int* cfg) {
    if (!h || !cfg) return LB_ERR_ARG;
    if (sweep_config(h, &cfg[0], &cfg[1], &cfg[2], &cfg[3]) < 0) return LB_ERR_STATE;
    return LB_OK;
}

int lb_cluster_info(lb_handle* h, int* nblocks, int* max_levels) {
    if (!h || !nblocks || !max_levels) return LB_ERR_ARG;
    if (!h->angle_ready) return fail(h, LB_ERR_STATE, "lb_cluster_info: quadrature not set");
    *nblocks = h->nclusters;
    *max_levels = h->max_cluster_levels;
    return LB_OK;
}

int lb_cluster_layout(lb_handle* h, long long* rec_base, int* blk_elem, int* max_records) {
    if (!h || !rec_base || !max_records) return LB_ERR_ARG;
    if (!h->angle_ready) return fail(h, LB_ERR_STATE, "lb_cluster_layout: quadrature not set");
    if (h->nclusters <= 0) return fail(h, LB_ERR_STATE, "lb_cluster_layout: the mesh has no block schedule");
    std::copy(h->crec_base_h.begin(), h->crec_base_h.end(), rec_base);
    *max_records = h->max_cluster_records;
    if (blk_elem) {
        if (h->blk_elem_h.empty())
            for (int q = 0; q < h->nclusters * kClusterSize; ++q) blk_elem[q] = q < h->NE ? q : -1;
        else
            std::copy(h->blk_elem_h.begin(), h->blk_elem_h.end(), blk_elem);
    }
    return LB_OK;
}

int lb_get_cluster_schedule(lb_handle* h, int* rec, int* starts, int* nlevels) {
    if (!h || !rec || !starts || !nlevels) return LB_ERR_ARG;
    if (!h->angle_ready) return fail(h, LB_ERR_STATE, "lb_get_cluster_schedule: quadrature not set");
    if (h->nclusters <= 0) return fail(h, LB_ERR_STATE, "lb_get_cluster_schedule: the mesh has no block schedule");
    const size_t n = (size_t)h->crec_base_h[h->NI];
    if (h->device < 0) {
        std::memcpy(rec, h->crec_h.data(), sizeof(int4) * n);
    } else {
        cudaSetDevice(h->device);
        cudaError_t e = cudaMemcpy(rec, h->d_crec, sizeof(int4) * n, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_fail(h, e, "lb_get_cluster_schedule");
    }
    const size_t ld = (size_t)h->max_cluster_records + 1;
    for (int i = 0; i < h->NI; ++i) {
        nlevels[i] = h->ncl_h[i];
        for (int L = 0; L <= h->ncl_h[i]; ++L) starts[(size_t)i * ld + L] = h->cl_start_h[h->cl_base_h[i] + L];
    }
    return LB_OK;
}

int lb_givens(double x, double y, double* c, double* s, double* r) {
    if (!c || !s || !r) return LB_ERR_ARG;
    givens_rotation(x, y, *c, *s);
    *r = x;
    return LB_OK;
}

int lb_mesh_types(lb_handle* h, int* ntypes) {
    if (!h || !ntypes) return LB_ERR_ARG;
    if (!h->mesh_ready) return fail(h, LB_ERR_STATE, "lb_mesh_types: mesh not set");
    *ntypes = h->ngeom;
    return LB_OK;
}

int lb_synchronize(lb_handle* h) {
    if (!h) return LB_ERR_ARG;
    if (h->device < 0) return LB_OK;
    cudaSetDevice(h->device);
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "synchronize");
    return moments_tc_status(h);
}

int lb_probe_pipeline_timeout(lb_handle* h, long long polls) {
    if (!h || polls < 1) return LB_ERR_ARG;
    if (h->device < 0) return fail(h, LB_ERR_STATE, "host-only handle: no device attached");
    cudaSetDevice(h->device);
    return tc_wait_probe(h, polls);
}

}  // extern "C"
