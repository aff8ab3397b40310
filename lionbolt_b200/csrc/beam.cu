// Uncollided fluence of a planar beam (the first-collision source data) on the device.
//
// Reference: Lionbolt ray-traces every quadrature point of every element in the beam back to the beam
// plane (RayTracing.f90:152-201), intersecting the segment with every region-boundary face
// (TraceVector, RayTracing.f90:205-379: O(rays x region faces)) to get per-material path lengths,
// applies Beer's law (FluenceQuadrature.f90:28-32) and projects the quadrature values onto the
// element's linear DG basis with the inverse mass matrix (FCSSource.f90:134-169; the same values are
// added to the group's fluence by AddAngularFluence.f90:109-166).
//
// Here one thread takes one (element, quadrature point) and walks the ray tet to tet through face
// neighbours in FP64, accumulating sigma_t * length of every tet it crosses until it reaches the beam
// plane or leaves the mesh: O(tets crossed) per ray instead of O(region faces), and the sum is the
// optical depth directly.  The four threads of an element combine their values with warp shuffles:
// with the 4-point rule (barycentric a on the point's vertex, b on the others, weights 1/24 on the
// reference tet) the projection M^-1 sum_q w_q N_k(q) phi_q is c_k = sqrt(5) phi_k + (1 - sqrt(5))/4
// sum_q phi_q (point k nearest vertex k).
#include "lb_internal.h"
#include <cmath>
#include <cstring>

namespace lb {
namespace {

constexpr double kQA = 0.58541019662496845446;   // (5 + 3 sqrt 5) / 20
constexpr double kQB = 0.13819660112501051518;   // (5 - sqrt 5) / 20
constexpr double kSqrt5 = 2.2360679774997896964;
constexpr double kInFieldTol = 1e-12;            // InField.f90:16

struct BeamArgs {
    const double* __restrict__ xyz;     // [NN][3]
    const int* __restrict__ node;       // [NE][4]
    const int* __restrict__ nbr;        // [NE][4], -1 on the boundary
    const int* __restrict__ mat;        // [NE]
    const double4* __restrict__ plane;  // [NE][4] outward unit normal and offset n . x of each face
    const double* __restrict__ attn;    // [Nm] total cross sections of the beam's group
    double* __restrict__ unc;           // [NE][4] DG coefficients of the uncollided fluence
    int* __restrict__ stuck;            // rays whose walk hit the step limit
    double ox, oy, oz;                  // beam origin
    double ax, ay, az;                  // beam axis (unit)
    double e1x, e1y, e1z, e2x, e2y, e2z;   // unit vectors spanning the beam plane
    double hw1, hw2;                    // half widths of the rectangular field along e1, e2
    int NE;
    int max_steps;
};

__global__ void __launch_bounds__(256) beam_uncollided_kernel(BeamArgs a) {
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int e = (int)(tid >> 2), q = (int)(tid & 3);
    const bool live = e < a.NE;
    double phi = 0.0;
    if (live) {
        // quadrature point q (barycentric kQA on vertex q)
        double x = 0.0, y = 0.0, z = 0.0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int v = __ldg(&a.node[4 * e + k]);
            const double c = k == q ? kQA : kQB;
            x = fma(c, __ldg(&a.xyz[3 * v]), x);
            y = fma(c, __ldg(&a.xyz[3 * v + 1]), y);
            z = fma(c, __ldg(&a.xyz[3 * v + 2]), z);
        }
        // InField (rectangle): the part of x - origin perpendicular to the axis, along e1 and e2
        const double ux = x - a.ox, uy = y - a.oy, uz = z - a.oz;
        const double ua = ux * a.ax + uy * a.ay + uz * a.az;
        const double vx = ux - ua * a.ax, vy = uy - ua * a.ay, vz = uz - ua * a.az;
        const double s1 = vx * a.e1x + vy * a.e1y + vz * a.e1z;
        const double s2 = vx * a.e2x + vy * a.e2y + vz * a.e2z;
        if (fabs(s1) <= a.hw1 + kInFieldTol && fabs(s2) <= a.hw2 + kInFieldTol) {
            // walk from x towards its projection Rp = origin + s1' e1 + s2' e2 on the beam plane
            const double p1 = ux * a.e1x + uy * a.e1y + uz * a.e1z;
            const double p2 = ux * a.e2x + uy * a.e2y + uz * a.e2z;
            double dx = a.ox + p1 * a.e1x + p2 * a.e2x - x;
            double dy = a.oy + p1 * a.e1y + p2 * a.e2y - y;
            double dz = a.oz + p1 * a.e1z + p2 * a.e2z - z;
            double remaining = sqrt(dx * dx + dy * dy + dz * dz);
            double tau = 0.0;
            if (remaining > 0.0) {
                const double il = 1.0 / remaining;
                dx *= il;
                dy *= il;
                dz *= il;
                int cur = e, steps = 0;
                while (cur >= 0) {
                    // exit face: the nearest face plane ahead of the ray
                    double tmin = 1e300;
                    int fexit = -1;
#pragma unroll
                    for (int f = 0; f < 4; ++f) {
                        const double4 pl = a.plane[4 * cur + f];
                        const double den = pl.x * dx + pl.y * dy + pl.z * dz;
                        if (den > 0.0) {
                            const double t = (pl.w - (pl.x * x + pl.y * y + pl.z * z)) / den;
                            if (t < tmin) {
                                tmin = t;
                                fexit = f;
                            }
                        }
                    }
                    if (fexit < 0) break;
                    const double seg = fmin(fmax(tmin, 0.0), remaining);
                    tau = fma(__ldg(&a.attn[__ldg(&a.mat[cur])]), seg, tau);
                    remaining -= seg;
                    if (remaining <= 0.0) break;
                    x = fma(seg, dx, x);
                    y = fma(seg, dy, y);
                    z = fma(seg, dz, z);
                    cur = __ldg(&a.nbr[4 * cur + fexit]);
                    if (++steps > a.max_steps) {
                        atomicAdd(a.stuck, 1);
                        tau = 0.0;
                        break;
                    }
                }
            }
            phi = exp(-tau);   // Beer's law, FluenceQuadrature.f90:28-32
        }
    }
    // L2 projection onto the element's linear DG basis (the element's four lanes are adjacent)
    const unsigned mask = 0xFFFFFFFFu;
    double sum = phi + __shfl_xor_sync(mask, phi, 1);
    sum += __shfl_xor_sync(mask, sum, 2);
    if (live) a.unc[4 * (size_t)e + q] = kSqrt5 * phi + 0.25 * (1.0 - kSqrt5) * sum;
}

}  // namespace

// Face planes, coordinates, connectivity and neighbours of the mesh on the device (built on first use).
static int beam_prepare(Handle* h) {
    if (h->beam_mesh_version == h->mesh_version && h->d_beam_plane) return LB_OK;
    for (void** p : {(void**)&h->d_beam_plane, (void**)&h->d_beam_xyz, (void**)&h->d_beam_node, (void**)&h->d_beam_nbr})
        if (*p) {
            cudaFree(*p);
            *p = nullptr;
        }
    static const int F2K[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
    const int NE = h->NE;
    std::vector<double4> pl((size_t)NE * 4);
    for (int e = 0; e < NE; ++e)
        for (int f = 0; f < 4; ++f) {
            const double* n = &h->nrm[((size_t)e * 4 + f) * 3];
            const double* x = &h->rg[(size_t)h->node[(size_t)e * 4 + F2K[f][0]] * 3];
            pl[(size_t)e * 4 + f] = make_double4(n[0], n[1], n[2], n[0] * x[0] + n[1] * x[1] + n[2] * x[2]);
        }
    auto up = [&](void** p, const void* src, size_t bytes, const char* what) -> int {
        cudaError_t err = cudaMalloc(p, bytes);
        if (err == cudaSuccess) err = cudaMemcpy(*p, src, bytes, cudaMemcpyHostToDevice);
        return err == cudaSuccess ? LB_OK : cuda_fail(h, err, what);
    };
    int rc = up((void**)&h->d_beam_plane, pl.data(), sizeof(double4) * pl.size(), "beam: face planes");
    if (!rc) rc = up((void**)&h->d_beam_xyz, h->rg.data(), sizeof(double) * h->rg.size(), "beam: coordinates");
    if (!rc) rc = up((void**)&h->d_beam_node, h->node.data(), sizeof(int) * h->node.size(), "beam: connectivity");
    if (!rc) rc = up((void**)&h->d_beam_nbr, h->nbr.data(), sizeof(int) * h->nbr.size(), "beam: neighbours");
    if (rc) return rc;
    h->beam_mesh_version = h->mesh_version;
    return LB_OK;
}

}  // namespace lb

using namespace lb;

extern "C" int lb_beam_uncollided(lb_handle* hh, const double* origin, const double* axis, const double* e1,
                                  const double* e2, double width1, double width2, const double* attn,
                                  double* unc) {
    Handle* h = reinterpret_cast<Handle*>(hh);
    if (!h || !origin || !axis || !e1 || !e2 || !attn) return LB_ERR_ARG;
    if (h->device < 0) return fail(h, LB_ERR_STATE, "host-only handle: no device attached");
    if (!h->mesh_ready) return fail(h, LB_ERR_STATE, "lb_beam_uncollided: mesh not set");
    if (!(width1 >= 0.0) || !(width2 >= 0.0)) return fail(h, LB_ERR_ARG, "lb_beam_uncollided: negative field width");
    for (int m = 0; m < h->Nm; ++m)
        if (!std::isfinite(attn[m]) || attn[m] < 0.0) return fail(h, LB_ERR_NAN, "lb_beam_uncollided: bad cross section");
    cudaSetDevice(h->device);
    int rc = beam_prepare(h);
    if (rc) return rc;
    const size_t NENK = (size_t)h->NENK;
    double* d_attn = nullptr;
    int* d_stuck = nullptr;
    cudaError_t e = cudaMalloc(&d_attn, sizeof(double) * h->Nm);
    if (e == cudaSuccess) e = cudaMalloc(&d_stuck, sizeof(int));
    if (e == cudaSuccess && !h->d_unc) e = cudaMalloc(&h->d_unc, sizeof(double) * NENK);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_attn, attn, sizeof(double) * h->Nm, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_stuck, 0, sizeof(int), h->stream);
    if (e != cudaSuccess) {
        cudaFree(d_attn);
        cudaFree(d_stuck);
        return cuda_fail(h, e, "lb_beam_uncollided: buffers");
    }
    BeamArgs a{};
    a.xyz = h->d_beam_xyz;
    a.node = h->d_beam_node;
    a.nbr = h->d_beam_nbr;
    a.mat = h->d_mat;
    a.plane = h->d_beam_plane;
    a.attn = d_attn;
    a.unc = h->d_unc;
    a.stuck = d_stuck;
    a.ox = origin[0]; a.oy = origin[1]; a.oz = origin[2];
    a.ax = axis[0]; a.ay = axis[1]; a.az = axis[2];
    a.e1x = e1[0]; a.e1y = e1[1]; a.e1z = e1[2];
    a.e2x = e2[0]; a.e2y = e2[1]; a.e2z = e2[2];
    a.hw1 = 0.5 * width1;
    a.hw2 = 0.5 * width2;
    a.NE = h->NE;
    a.max_steps = 4 * h->NE + 64;
    Timer t;
    timer_begin(h, LB_T_TALLY, t);
    const long long threads = 4LL * h->NE;
    beam_uncollided_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, h->stream>>>(a);
    timer_end(h, t);
    e = cudaGetLastError();
    int stuck = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&stuck, d_stuck, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess && unc) e = cudaMemcpyAsync(unc, h->d_unc, sizeof(double) * NENK, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(d_attn);
    cudaFree(d_stuck);
    if (e != cudaSuccess) return cuda_fail(h, e, "lb_beam_uncollided");
    if (stuck) return fail(h, LB_ERR_STATE, "lb_beam_uncollided: a ray walk did not reach the beam plane");
    return LB_OK;
}
