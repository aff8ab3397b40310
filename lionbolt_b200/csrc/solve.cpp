// Operator applications and Krylov drivers in flux-moment space.
//
// Reference algorithm: BoltzmannOp%MatInv (BoltzmannOperator.f90:106-151) solves
// (I - T^{-1}K) psi = T^{-1} q with SPARSKIT GMRES(m) on the full angular flux
// (n = NENK*NI, iters.f:1901-2206) or with source iteration (SourceIteration.f90).
// Here K = M Sigma D (exact, see moments.cu), so with phi = D psi the same fixed point solves
//   A phi = (I - D T^{-1} M Sigma) phi = b,   b = D T^{-1} q,
// and psi = T^{-1}(M Sigma phi + q).  The Krylov vectors shrink from NI*NENK to nm*NENK
// (288 -> 36 per node at P5) and stay FP64; the sweep and the moment GEMMs run in FP32.
// The Arnoldi/Givens/restart logic and the stopping test ||b - A phi|| <= rtol||b|| + atol follow
// the reference's SPARSKIT gmres/fgmres; orthogonalisation is Gram-corrected classical
// Gram-Schmidt (two fused passes over the basis per Arnoldi step, see gmres_device).
#include "lb_internal.h"
#include "gmres_host.h"
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <omp.h>

namespace lb {

int k_multi_axpy_norm(Handle* h, double* w, const double* V, size_t ldv, int nv, const double* coef, size_t n, double* nrm2);

static int need_ready(Handle* h, bool phys = true) {
    if (h->device < 0) return fail(h, LB_ERR_STATE, "host-only handle: no device attached");
    if (!h->mesh_ready || !h->angle_ready || (phys && !h->phys_ready))
        return fail(h, LB_ERR_STATE, "operator was called, but the operator was not ready");
    return LB_OK;
}

int ensure_krylov(Handle* h, int m, bool flexible) {
    size_t n = (size_t)h->nm * (size_t)h->NENK;
    bool realloc_v = (h->kry_n != n) || (h->kry_m < m) || !h->d_V;
    if (realloc_v) {
        if (h->d_V) cudaFree(h->d_V);
        if (h->d_x) cudaFree(h->d_x);
        if (h->d_b) cudaFree(h->d_b);
        if (h->d_t) cudaFree(h->d_t);
        if (h->d_Z) { cudaFree(h->d_Z); h->d_Z = nullptr; }
        h->d_V = h->d_x = h->d_b = h->d_t = nullptr;
        cudaError_t e = cudaMalloc(&h->d_V, sizeof(double) * n * (size_t)(m + 1));
        if (e == cudaSuccess) e = cudaMalloc(&h->d_x, sizeof(double) * n);
        if (e == cudaSuccess) e = cudaMalloc(&h->d_b, sizeof(double) * n);
        if (e == cudaSuccess) e = cudaMalloc(&h->d_t, sizeof(double) * n);
        if (e != cudaSuccess) return cuda_fail(h, e, "Krylov workspace");
        h->kry_n = n;
        h->kry_m = m;
    }
    if (!h->d_red) {
        cudaError_t e = cudaMalloc(&h->d_red, sizeof(double) * 65536);
        if (e != cudaSuccess) return cuda_fail(h, e, "reduction buffer");
    }
    if (flexible && !h->d_Z) {
        cudaError_t e = cudaMalloc(&h->d_Z, sizeof(double) * n * (size_t)h->kry_m);
        if (e != cudaSuccess) return cuda_fail(h, e, "FGMRES workspace");
    }
    return LB_OK;
}

// y = A x = x - D T^{-1} M Sigma x   (sigl: per-material sigma_l table, within group)
static int apply_A(Handle* h, const double* x, double* y, const float* sigl) {
    int rc = launch_m2d(h, x, sigl, nullptr, nullptr, h->d_psi);
    if (!rc) rc = launch_sweep(h, h->d_psi);
    if (!rc) rc = launch_d2m(h, h->d_psi, x, 1.0, -1.0, y);
    return rc;
}

// z = D T^{-1} M Sigma x, so that A x = x - z: the Arnoldi step forms the difference in its projection passes,
// which read x (the last basis vector) anyway, and the D2M epilogue skips reading x.
static int apply_Z(Handle* h, const double* x, double* z, const float* sigl) {
    int rc = launch_m2d(h, x, sigl, nullptr, nullptr, h->d_psi);
    if (!rc) rc = launch_sweep(h, h->d_psi);
    if (!rc) rc = launch_d2m(h, h->d_psi, nullptr, 0.0, 1.0, z);
    return rc;
}

// y = D T^{-1} (M (Sigma x + a) + qext)   (any of x, a, qext may be null)
static int apply_transport_moments(Handle* h, const double* x, const float* sigl, const double* a, const float* qext,
                                   double* y) {
    int rc;
    if (!x && !a) {
        if (!qext) return fail(h, LB_ERR_ARG, "empty source");
        cudaError_t e = cudaMemcpyAsync(h->d_psi, qext, sizeof(float) * h->psi_elems, cudaMemcpyDeviceToDevice, h->stream);
        if (e != cudaSuccess) return cuda_fail(h, e, "copy source");
        rc = LB_OK;
    } else {
        rc = launch_m2d(h, x, sigl, a, qext, h->d_psi);
    }
    if (!rc) rc = launch_sweep(h, h->d_psi);
    if (!rc) rc = launch_d2m(h, h->d_psi, nullptr, 0.0, 1.0, y);
    return rc;
}

static double vnorm(Handle* h, const double* v, size_t n, int* rc) {
    double s = 0.0;
    *rc = k_dots(h, v, n, 1, v, n, &s);
    return std::sqrt(s);
}

struct KrylovResult {
    int status = LB_OK;
    int nmv = 0;
    double resid = 0.0;
};

using DevOp = std::function<int(const double* in, double* out)>;
// Right preconditioner: out = P(in), with in * scale the normalised basis vector (P may use it to fix
// the magnitude of its input; a linear P ignores it).
using PrecOp = std::function<int(const double* in, double scale, double* out)>;

// Restarted GMRES(m) / FGMRES(m) (right preconditioner `prec`), SPARSKIT semantics.
// matvec_z (plain GMRES only): z with A x = x - z, used by the Arnoldi steps (see apply_Z); the residual at a
// (re)start still uses matvec.
static KrylovResult gmres_device(Handle* h, size_t n, const double* rhs, double* sol, int m, double rtol, double atol,
                                 int maxit, const DevOp& matvec, const PrecOp* prec, const DevOp* matvec_z = nullptr) {
    KrylovResult res;
    int rc = 0;
    double* V = h->d_V;
    double* Z = h->d_Z;
    GmresHost gh(m);
    std::vector<double> hh(m + 2), h2(m + 2), cc(m + 2), cw(m + 2), coef;
    // The stored basis vectors W_i are not normalised: V_i = sc[i] W_i.  The scale factors enter the
    // coefficients of every pass instead, which saves the two full-vector passes of a normalisation
    // (v0 = r / alpha, v_k = w / h_k) per Arnoldi step.  The (flexible) Z_i are stored the same way.
    std::vector<double> sc(m + 2, 1.0);
    const int ldg = m + 2;
    std::vector<double> G((size_t)ldg * ldg, 0.0);   // Gram matrix V^T V of the current cycle's basis
    double rn = vnorm(h, rhs, n, &rc);
    if (rc) { res.status = rc; return res; }
    const double fpar4 = rtol * rn + atol;
    double fpar5 = 0.0;
    int nmv = 0;
    // Stagnation: the operator applies FP32 sweeps, so a tolerance below what they resolve leaves the true
    // residual at a floor while the cycle's residual estimate keeps reaching the target; five restarts in a
    // row that do not lower the true residual by 1 % end the solve instead of cycling without end.
    double best = HUGE_VAL;
    int stalled = 0;
    while (true) {
        // r = rhs - A sol
        if ((rc = matvec(sol, V))) { res.status = rc; return res; }
        ++nmv;
        double alpha = 0.0;
        if ((rc = k_axpby_norm(h, V, rhs, 1.0, -1.0, n, &alpha))) { res.status = rc; return res; }   // V0 = rhs - V0
        alpha = std::sqrt(alpha);
        if (std::isnan(alpha)) { res.status = fail(h, LB_ERR_NAN, "RESIDUAL NORM is NaN."); return res; }
        fpar5 = alpha;
        gh.start(alpha);
        if (alpha <= fpar4) { res.status = LB_OK; res.nmv = nmv; res.resid = alpha; return res; }
        if (alpha < 0.99 * best) {
            best = alpha;
            stalled = 0;
        } else if (++stalled >= 5) {
            char msg[200];
            std::snprintf(msg, sizeof msg,
                          "GMRES stagnated: the true residual stays at %.3e against a target of %.3e (below what the "
                          "FP32 sweep resolves)", alpha, fpar4);
            res.status = fail(h, LB_ERR_NOCONV, msg);
            res.nmv = nmv;
            res.resid = alpha;
            return res;
        }
        sc[0] = 1.0 / alpha;
        G[0] = 1.0;
        int k = 0;
        bool breakdown = false;
        while (true) {
            ++k;
            const double* vin = V + (size_t)(k - 1) * n;
            if (prec) {
                if ((rc = (*prec)(vin, sc[k - 1], Z + (size_t)(k - 1) * n))) { res.status = rc; return res; }
                vin = Z + (size_t)(k - 1) * n;
            }
            double* vk = V + (size_t)k * n;
            const bool zm = matvec_z && !prec;   // vk holds z; A v = V_{k-1} - z is formed by the passes
            if ((rc = zm ? (*matvec_z)(vin, vk) : matvec(vin, vk))) { res.status = rc; return res; }
            ++nmv;
            // Gram-corrected classical Gram-Schmidt in two passes over V[0..k-1]: (1) hh = V^T vk and
            // |vk|^2;  (2) vk -= V c with G c = hh (G = V^T V, kept up to date from the dots of pass 2),
            // with h2 = V^T vk and |vk|^2 of the result in the same pass;  then vk /= hk.  Then
            // A v_{k-1} = V c + hk v_k holds exactly, hk is a measured norm, and the residual
            // non-orthogonality h2 / hk enters G for the next steps (this replaces the second projection
            // pass of classical Gram-Schmidt with re-orthogonalisation: 2k + 5 vector passes per step
            // instead of 3k + 5).
            // (vk holds A W_{k-1} = A V_{k-1} / sc[k-1]; the dots below are of the stored vectors)
            const double s1 = sc[k - 1];
            double nrm0 = 0.0, nrm1 = 0.0;
            if ((rc = k_dots_norm(h, V, n, k, vk, n, hh.data(), &nrm0, zm))) { res.status = rc; return res; }
            for (int i = 0; i < k; ++i) hh[i] *= sc[i] * s1;
            if (!gram_solve(G, ldg, k, hh.data(), cc.data()))
                for (int i = 0; i < k; ++i) cc[i] = hh[i];
            for (int i = 0; i < k; ++i) cw[i] = cc[i] * sc[i] / s1;
            if ((rc = k_axpy_dots(h, vk, V, n, k, cw.data(), n, h2.data(), &nrm1, zm))) { res.status = rc; return res; }
            for (int i = 0; i < k; ++i) {
                hh[i] = cc[i];
                h2[i] *= sc[i] * s1;
            }
            const double hk = s1 * std::sqrt(std::max(0.0, nrm1));
            if (std::isnan(hk)) { res.status = fail(h, LB_ERR_NAN, "RESIDUAL NORM is NaN."); return res; }
            if (!(hk > 0.0)) {
                for (int i = 0; i < k; ++i) gh.H[k][i + 1] = hh[i];
                gh.H[k][k + 1] = hk;
                breakdown = true;
                --k;
                break;
            }
            sc[k] = s1 / hk;
            for (int i = 0; i < k; ++i) G[(size_t)i * ldg + k] = G[(size_t)k * ldg + i] = h2[i] / hk;
            G[(size_t)k * ldg + k] = 1.0;
            alpha = gh.add_column(k, hh.data(), hk);
            fpar5 = alpha;
            if (k < m && !(alpha <= fpar4) && (maxit <= 0 || nmv < maxit)) continue;
            break;
        }
        const int kk = gh.solve(k, coef);
        if (kk == 0) {
            if (breakdown) continue;   // nothing new in the basis: recompute the true residual
            res.status = fail(h, LB_ERR_BREAKDOWN, "GMRES : Anticipated breakdown / division by zero.");
            return res;
        }
        // sol += sum_i y_i V_i (or Z_i): multi-axpy with negated coefficients, on the stored vectors
        for (int i = 0; i < kk; ++i) coef[i] *= sc[i];
        if ((rc = k_multi_axpy(h, sol, prec ? Z : V, n, kk, coef.data(), n))) { res.status = rc; return res; }
        if (breakdown) continue;
        if ((nmv < maxit || maxit <= 0) && fpar5 > fpar4) continue;
        res.nmv = nmv;
        res.resid = fpar5;
        if (fpar5 <= fpar4) {
            res.status = LB_OK;
        } else {
            res.status = fail(h, LB_ERR_NOCONV, "GMRES : Iteration did not converge in specified iteration limits.");
        }
        return res;
    }
}

// Source iteration (SourceIteration.f90:33-80) in moment space: phi = b; w = b;
// repeat w <- D T^{-1} M Sigma w; phi += w until ||w|| <= atol + rtol ||b||.
static KrylovResult si_device(Handle* h, size_t n, const double* b, double* phi, double rtol, double atol, int maxit,
                              const float* sigl) {
    KrylovResult res;
    int rc = 0;
    double* w = h->d_t;
    k_copy(h, phi, b, n);
    k_copy(h, w, b, n);
    double norms = vnorm(h, b, n, &rc);
    int it = 1;
    if ((rc = apply_transport_moments(h, w, sigl, nullptr, nullptr, w))) { res.status = rc; return res; }
    k_axpby(h, phi, w, 1.0, 1.0, n);
    while (true) {
        ++it;
        double rn = vnorm(h, w, n, &rc);
        if (rc) { res.status = rc; return res; }
        res.resid = rn;
        res.nmv = it;
        if (std::isnan(rn)) { res.status = fail(h, LB_ERR_NAN, "RESIDUAL NORM is NaN."); return res; }
        if (rn <= atol + norms * rtol) return res;
        if (maxit > 0 && it > maxit) { res.status = fail(h, LB_ERR_NOCONV, "SI did not converge in the iteration limit"); return res; }
        if ((rc = apply_transport_moments(h, w, sigl, nullptr, nullptr, w))) { res.status = rc; return res; }
        k_axpby(h, phi, w, 1.0, 1.0, n);
    }
}

// Solve A phi = b in moment space with the selected solver; phi holds the initial guess.  budget > 0
// caps the learned path's FGMRES at that many operator applications before plain GMRES takes over.
static KrylovResult moment_solve(Handle* h, const double* b, double* phi, int solver, int m, double rtol, double atol,
                                 int maxit, const float* sigl, int budget = 0) {
    const size_t n = (size_t)h->nm * (size_t)h->NENK;
    if (solver == LB_SOLVER_SI) return si_device(h, n, b, phi, rtol, atol, maxit, sigl);
    DevOp mv = [h, sigl](const double* in, double* out) { return apply_A(h, in, out, sigl); };
    DevOp mz = [h, sigl](const double* in, double* out) { return apply_Z(h, in, out, sigl); };
    if (solver == LB_SOLVER_FGMRES) {
        // FGMRES(m) (iters.f:2511-2795) with the caller's per-moment diagonal as right preconditioner
        if (!h->pdiag.empty() && (int)h->pdiag.size() != h->nm) {
            KrylovResult bad;
            bad.status = fail(h, LB_ERR_ARG, "FGMRES: the diagonal preconditioner has another moment count");
            return bad;
        }
        const size_t NENK = (size_t)h->NENK;
        PrecOp pc = [h, NENK, n](const double* in, double, double* out) {
            if (h->pdiag.empty()) return k_copy(h, out, in, n);
            return k_scale_rows(h, out, in, h->pdiag.data(), h->nm, NENK);
        };
        return gmres_device(h, n, b, phi, m, rtol, atol, maxit, mv, &pc);
    }
    if (solver == LB_SOLVER_FGMRES_ML) {
        if (!mlp_ready(h)) {
            // plain GMRES is the fallback when no trained network is loaded
            return gmres_device(h, n, b, phi, m, rtol, atol, maxit, mv, nullptr, &mz);
        }
        // Learned path: FGMRES(m) with the network as right preconditioner, capped at `budget` operator
        // applications (plain GMRES's count on this group in calibration), else 4m, and never beyond
        // the caller's limit.
        PrecOp pc = [h](const double* in, double scale, double* out) { return mlp_apply_precond(h, in, out, scale); };
        int cap = budget > 0 ? budget : 4 * m;
        if (maxit > 0) cap = std::min(cap, maxit);
        KrylovResult kr = gmres_device(h, n, b, phi, m, rtol, atol, cap, mv, &pc);
        if (kr.status != LB_OK && kr.status != LB_ERR_NOCONV && kr.status != LB_ERR_BREAKDOWN &&
            kr.status != LB_ERR_NAN)
            return kr;   // CUDA or argument errors end the solve
        int nmv = kr.nmv;
        int rc = 0;
        if (kr.status == LB_ERR_NAN) {
            k_copy(h, phi, b, n);   // the learned iterate is unusable: restart from the first-flight moments
        } else {
            // Plain-operator check: the true residual ||b - A phi|| of the learned iterate.
            if ((rc = apply_A(h, phi, h->d_t, sigl))) { kr.status = rc; return kr; }
            ++nmv;
            double rn = 0.0;
            if ((rc = k_axpby_norm(h, h->d_t, b, 1.0, -1.0, n, &rn))) { kr.status = rc; return kr; }
            rn = std::sqrt(rn);
            const double bn = vnorm(h, b, n, &rc);
            if (rc) { kr.status = rc; return kr; }
            if (rn <= rtol * bn + atol) {
                h->err.clear();
                kr.status = LB_OK;
                kr.nmv = nmv;
                kr.resid = rn;
                return kr;
            }
        }
        // Fallback: plain GMRES(m) from the learned iterate, under the caller's limit.
        h->err.clear();
        KrylovResult k2 = gmres_device(h, n, b, phi, m, rtol, atol, maxit > 0 ? std::max(1, maxit - nmv) : 0, mv,
                                       nullptr, &mz);
        k2.nmv += nmv;
        return k2;
    }
    return gmres_device(h, n, b, phi, m, rtol, atol, maxit, mv, nullptr, &mz);
}

// ---------------------------------------------------------------------------------------------
//  angular <-> device transfers (FP64 host, FP32 device), chunked through a pinned staging area
// ---------------------------------------------------------------------------------------------
static int upload_angular(Handle* h, const double* hs, float* d) {
    const size_t total = h->psi_elems;
    const size_t chunk = (size_t)1 << 24;
    double* stage = nullptr;
    cudaError_t e = cudaMalloc(&stage, sizeof(double) * std::min(total, chunk));
    if (e != cudaSuccess) return cuda_fail(h, e, "staging buffer");
    for (size_t o = 0; o < total; o += chunk) {
        size_t c = std::min(chunk, total - o);
        e = cudaMemcpyAsync(stage, hs + o, sizeof(double) * c, cudaMemcpyHostToDevice, h->stream);
        if (e != cudaSuccess) break;
        k_f64_to_f32(h, d + o, stage, c);
        e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) break;
    }
    cudaFree(stage);
    return e == cudaSuccess ? LB_OK : cuda_fail(h, e, "upload angular vector");
}

static int download_angular(Handle* h, const float* d, double* hs) {
    const size_t total = h->psi_elems;
    const size_t chunk = (size_t)1 << 24;
    double* stage = nullptr;
    cudaError_t e = cudaMalloc(&stage, sizeof(double) * std::min(total, chunk));
    if (e != cudaSuccess) return cuda_fail(h, e, "staging buffer");
    for (size_t o = 0; o < total; o += chunk) {
        size_t c = std::min(chunk, total - o);
        k_f32_to_f64(h, stage, d + o, c);
        e = cudaMemcpyAsync(hs + o, stage, sizeof(double) * c, cudaMemcpyDeviceToHost, h->stream);
        if (e != cudaSuccess) break;
        e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) break;
    }
    cudaFree(stage);
    return e == cudaSuccess ? LB_OK : cuda_fail(h, e, "download angular vector");
}


}  // namespace lb

struct lb_handle : public lb::Handle {};

namespace lb {

// ---------------------------------------------------------------------------------------------
//  multigroup helpers (group loop of Main.f90:326-476)
// ---------------------------------------------------------------------------------------------
float* mg_table(Handle* h, int gp, int g) {
    return h->d_sigl_mg + (((size_t)gp * h->G + g) * h->Nm) * h->nmpad;
}

// Beam-direction harmonics Y_j(Omega_b) for the first-collision source.
void mg_prepare(Handle* h) {
    std::vector<double> yb(h->nm);
    real_sh(h->Ls, h->beam_dir.data(), yb.data());
    cudaMemcpyAsync(h->d_yb, yb.data(), sizeof(double) * h->nm, cudaMemcpyHostToDevice, h->stream);
    cudaStreamSynchronize(h->stream);
}

// Source and operator of group g from the solved groups g' < g in d_phi_all:
// d_src = sum_{g'<g} Sigma_{g'->g} phi_{g'} + first collision of the beam, and the within-group
// cross sections of g set on the handle.
int mg_group_sources(Handle* h, int g) {
    const int G = h->G, Nm = h->Nm, Ls = h->Ls, nm = h->nm, nmpad = h->nmpad;
    k_group_source(h, h->d_src, h->d_phi_all, h->d_sigl_mg, G, g, h->d_unc, h->d_yb, h->d_mat, h->NENK, Nm, nm,
                   nmpad);
    std::vector<double> st(h->mg_sigt.begin() + (size_t)g * Nm, h->mg_sigt.begin() + (size_t)(g + 1) * Nm);
    std::vector<double> ss((size_t)Nm * (Ls + 1));
    for (int mm = 0; mm < Nm; ++mm)
        for (int l = 0; l <= Ls; ++l)
            ss[(size_t)mm * (Ls + 1) + l] = h->mg_sigs[(((size_t)g * G + g) * Nm + mm) * (Ls + 1) + l];
    return lb_set_xs(static_cast<lb_handle*>(h), Ls, st.data(), ss.data());
}

// ... and d_b = D T^{-1} M d_src.
static int mg_group_setup(Handle* h, int g) {
    int rc = mg_group_sources(h, g);
    if (rc) return rc;
    return apply_transport_moments(h, nullptr, nullptr, h->d_src, nullptr, h->d_b);
}

}  // namespace lb

using namespace lb;

extern "C" {

int lb_transport_inv(lb_handle* h, double* s) {
    if (!h || !s) return LB_ERR_ARG;
    int rc = need_ready(h, false);
    if (rc) return rc;
    if (h->sigt.empty()) return fail(h, LB_ERR_STATE, "lb_transport_inv: cross sections not set");
    cudaSetDevice(h->device);
    if ((rc = upload_angular(h, s, h->d_psi))) return rc;
    if ((rc = launch_sweep(h, h->d_psi))) return rc;
    return download_angular(h, h->d_psi, s);
}

int lb_m2d_device(lb_handle* h, const double* phi, float* psi) {
    if (!h || !phi || !psi) return LB_ERR_ARG;
    int rc = need_ready(h);
    if (rc) return rc;
    cudaSetDevice(h->device);
    return launch_m2d(h, phi, h->d_sigl, nullptr, nullptr, psi);
}

int lb_d2m_device(lb_handle* h, const float* psi, double* phi) {
    if (!h || !phi || !psi) return LB_ERR_ARG;
    int rc = need_ready(h);
    if (rc) return rc;
    cudaSetDevice(h->device);
    return launch_d2m(h, psi, nullptr, 0.0, 1.0, phi);
}

int lb_scatter_apply(lb_handle* h, double* x) {
    if (!h || !x) return LB_ERR_ARG;
    int rc = need_ready(h);
    if (rc) return rc;
    cudaSetDevice(h->device);
    if ((rc = ensure_krylov(h, std::max(h->kry_m, 1), false))) return rc;
    if ((rc = upload_angular(h, x, h->d_psi))) return rc;
    if ((rc = launch_d2m(h, h->d_psi, nullptr, 0.0, 1.0, h->d_t))) return rc;
    if ((rc = launch_m2d(h, h->d_t, h->d_sigl, nullptr, nullptr, h->d_psi))) return rc;
    if ((rc = download_angular(h, h->d_psi, x))) return rc;
    return moments_tc_status(h);
}

int lb_boltzmann_matvec(lb_handle* h, double* x) {
    if (!h || !x) return LB_ERR_ARG;
    int rc = need_ready(h);
    if (rc) return rc;
    cudaSetDevice(h->device);
    if ((rc = ensure_krylov(h, std::max(h->kry_m, 1), false))) return rc;
    if ((rc = upload_angular(h, x, h->d_psi))) return rc;
    if ((rc = launch_d2m(h, h->d_psi, nullptr, 0.0, 1.0, h->d_t))) return rc;
    if ((rc = launch_m2d(h, h->d_t, h->d_sigl, nullptr, nullptr, h->d_psi))) return rc;
    if ((rc = launch_sweep(h, h->d_psi))) return rc;
    std::vector<double> y(h->psi_elems);
    if ((rc = download_angular(h, h->d_psi, y.data()))) return rc;
    if ((rc = moments_tc_status(h))) return rc;
#pragma omp parallel for schedule(static)
    for (size_t q = 0; q < y.size(); ++q) x[q] = x[q] - y[q];
    return LB_OK;
}

int lb_boltzmann_solve(lb_handle* h, double* s, int solver, int m, double rtol, double atol, int maxit, int* iters,
                       double* resid) {
    if (!h || !s) return LB_ERR_ARG;
    int rc = need_ready(h);
    if (rc) return rc;
    if (solver < 0 || solver > 3) return fail(h, LB_ERR_ARG, "unknown solver");
    if (m < 1) m = 10;
    if (m > 30) return fail(h, LB_ERR_ARG, "restart length must be <= 30");
    cudaSetDevice(h->device);
    if ((rc = ensure_krylov(h, m, solver == LB_SOLVER_FGMRES_ML || solver == LB_SOLVER_FGMRES))) return rc;
    if (!h->d_qext) {
        cudaError_t e = cudaMalloc(&h->d_qext, sizeof(float) * h->psi_elems);
        if (e != cudaSuccess) return cuda_fail(h, e, "angular source buffer");
    }
    if ((rc = upload_angular(h, s, h->d_qext))) return rc;
    const size_t n = h->kry_n;
    // b = D T^{-1} q
    if ((rc = apply_transport_moments(h, nullptr, nullptr, nullptr, h->d_qext, h->d_b))) return rc;
    k_copy(h, h->d_x, h->d_b, n);   // initial guess: the first-flight moments
    KrylovResult kr = moment_solve(h, h->d_b, h->d_x, solver, m, rtol, atol, maxit, h->d_sigl);
    if (iters) *iters = kr.nmv;
    if (resid) *resid = kr.resid;
    if (kr.status) return kr.status;
    // psi = T^{-1} (M Sigma phi + q)
    if ((rc = launch_m2d(h, h->d_x, h->d_sigl, nullptr, h->d_qext, h->d_psi))) return rc;
    if ((rc = launch_sweep(h, h->d_psi))) return rc;
    if ((rc = download_angular(h, h->d_psi, s))) return rc;
    return moments_tc_status(h);
}

int lb_set_right_precond_diag(lb_handle* h, int nm, const double* d) {
    if (!h || nm < 0 || nm > kMaxRowCoefs || (nm > 0 && !d)) return h ? fail(h, LB_ERR_ARG, "lb_set_right_precond_diag: bad arguments") : LB_ERR_ARG;
    if (nm == 0 || !d) h->pdiag.clear();
    else h->pdiag.assign(d, d + nm);
    return LB_OK;
}

int lb_mg_set_problem(lb_handle* h, int G, int Ls, const double* sigt, const double* sigs, const double* dd,
                      const double* unc, const double* beam_dir) {
    if (!h || G < 1 || !sigt || !sigs || !dd) return LB_ERR_ARG;
    if (h->device < 0) return fail(h, LB_ERR_STATE, "host-only handle: no device attached");
    if (!h->mesh_ready || !h->angle_ready) return fail(h, LB_ERR_STATE, "lb_mg_set_problem: mesh/quadrature not set");
    cudaSetDevice(h->device);
    const int Nm = h->Nm;
    h->G = G;
    h->mg_sigt.assign(sigt, sigt + (size_t)G * Nm);
    h->mg_sigs.assign(sigs, sigs + (size_t)G * G * Nm * (Ls + 1));
    h->mg_dd.assign(dd, dd + (size_t)G * Nm);
    h->beam_dir.assign(3, 0.0);
    if (beam_dir) h->beam_dir.assign(beam_dir, beam_dir + 3);
    // within-group XS of group 0 sets nm / the Y planes
    int rc = lb_set_xs(h, Ls, sigt, sigs);
    if (rc) return rc;
    const int nm = h->nm, nmpad = h->nmpad;
    // transfer tables sigma_l(j) for every (g', g) pair: [G][G][Nm][nmpad]
    std::vector<float> tab((size_t)G * G * Nm * nmpad, 0.f);
    for (int gp = 0; gp < G; ++gp)
        for (int g = 0; g < G; ++g)
            for (int m = 0; m < Nm; ++m)
                for (int l = 0; l <= Ls; ++l)
                    for (int j = l * l; j < (l + 1) * (l + 1); ++j)
                        tab[(((size_t)gp * G + g) * Nm + m) * nmpad + j] =
                            (float)sigs[(((size_t)gp * G + g) * Nm + m) * (Ls + 1) + l];
    const size_t NENK = (size_t)h->NENK;
    const bool same = h->mg_alloc_G == G && h->mg_alloc_nm == nm && h->mg_alloc_NENK == (long long)NENK &&
                      h->mg_alloc_tab == tab.size();
    if (!same) {
        auto realloc = [&](auto** p, size_t cnt, const char* what) -> int {
            if (*p) cudaFree(*p);
            *p = nullptr;
            cudaError_t ee = cudaMalloc((void**)p, sizeof(**p) * cnt);
            return ee == cudaSuccess ? LB_OK : cuda_fail(h, ee, what);
        };
        if ((rc = realloc(&h->d_sigl_mg, tab.size(), "transfer tables"))) return rc;
        if ((rc = realloc(&h->d_unc, NENK, "uncollided flux"))) return rc;
        if ((rc = realloc(&h->d_phi_all, (size_t)G * nm * NENK, "group flux moments"))) return rc;
        if ((rc = realloc(&h->d_src, (size_t)nm * NENK, "group source"))) return rc;
        if ((rc = realloc(&h->d_dose, NENK, "dose"))) return rc;
        if ((rc = realloc(&h->d_flux, (size_t)G * NENK, "group fluence"))) return rc;
        if ((rc = realloc(&h->d_yb, 256, "beam harmonics"))) return rc;
        if ((rc = realloc(&h->d_dd, (size_t)G * Nm, "dose cross sections"))) return rc;
        h->mg_alloc_G = G; h->mg_alloc_nm = nm; h->mg_alloc_NENK = (long long)NENK; h->mg_alloc_tab = tab.size();
    }
    cudaError_t e = cudaMemcpyAsync(h->d_sigl_mg, tab.data(), sizeof(float) * tab.size(), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->d_dd, dd, sizeof(double) * (size_t)G * Nm, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) {
        if (unc) e = cudaMemcpyAsync(h->d_unc, unc, sizeof(double) * NENK, cudaMemcpyHostToDevice, h->stream);
        else e = cudaMemsetAsync(h->d_unc, 0, sizeof(double) * NENK, h->stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "upload problem");
    return LB_OK;
}

int lb_mg_update_inputs(lb_handle* h, const double* sigt, const double* sigs, const double* dd, const double* unc,
                        const double* beam_dir) {
    if (!h || h->device < 0 || h->G < 1 || !h->d_phi_all) return h ? fail(h, LB_ERR_STATE, "lb_mg_update_inputs: problem not set") : LB_ERR_ARG;
    return lb_mg_set_problem(h, h->G, h->Ls, sigt, sigs, dd, unc, beam_dir);
}

int lb_mg_solve(lb_handle* h, int solver, int m, double rtol, double atol, int maxit, int* iters) {
    if (!h || h->device < 0 || h->G < 1 || !h->d_phi_all) return h ? fail(h, LB_ERR_STATE, "lb_mg_solve: problem not set") : LB_ERR_ARG;
    if (solver < 0 || solver > 3) return fail(h, LB_ERR_ARG, "unknown solver");
    if (m < 1) m = 10;
    if (m > 30) return fail(h, LB_ERR_ARG, "restart length must be <= 30");
    cudaSetDevice(h->device);
    const int G = h->G, Nm = h->Nm;
    int rc = ensure_krylov(h, m, solver == LB_SOLVER_FGMRES_ML || solver == LB_SOLVER_FGMRES);
    if (rc) return rc;
    const size_t NENK = (size_t)h->NENK, n = h->kry_n;
    mg_prepare(h);
    cudaMemsetAsync(h->d_dose, 0, sizeof(double) * NENK, h->stream);
    for (int g = 0; g < G; ++g) {
        if ((rc = mg_group_setup(h, g))) break;
        double* phi = h->d_phi_all + (size_t)g * n;
        k_copy(h, phi, h->d_b, n);
        int sv = solver, budget = 0;
        if (solver == LB_SOLVER_FGMRES_ML) {
            if (g < (int)h->lp_groups.size() && !h->lp_groups[g]) sv = LB_SOLVER_GMRES;   // gated off for this group
            if (g < (int)h->lp_budget.size()) budget = h->lp_budget[g];
        }
        KrylovResult kr = moment_solve(h, h->d_b, phi, sv, m, rtol, atol, maxit, mg_table(h, g, g), budget);
        if (iters) iters[g] = kr.nmv;
        if ((rc = kr.status)) break;
        k_dose_tally(h, phi, h->d_unc, g == 0 ? 1.0 : 0.0, h->d_dd + (size_t)g * Nm, h->d_mat,
                     h->d_flux + (size_t)g * NENK, h->d_dose, (long long)NENK);
    }
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (!rc && e != cudaSuccess) rc = cuda_fail(h, e, "multigroup solve");
    if (!rc) rc = moments_tc_status(h);
    return rc;
}

int lb_lp_set_groups(lb_handle* h, int G, const int* enabled, const int* budget) {
    if (!h || G < 0 || (G > 0 && !enabled)) return h ? fail(h, LB_ERR_ARG, "lb_lp_set_groups: bad arguments") : LB_ERR_ARG;
    h->lp_groups.assign(G, 1);
    h->lp_budget.assign(budget ? G : 0, 0);
    for (int g = 0; g < G; ++g) {
        h->lp_groups[g] = enabled[g] != 0;
        if (budget) h->lp_budget[g] = std::max(0, budget[g]);
    }
    return LB_OK;
}

int lb_lp_calibrate(lb_handle* h, int m, double rtol, int* plain_iters, int* learned_iters) {
    if (!h || h->device < 0 || h->G < 1 || !h->d_phi_all)
        return h ? fail(h, LB_ERR_STATE, "lb_lp_calibrate: multigroup problem not set") : LB_ERR_ARG;
    if (!mlp_ready(h)) return fail(h, LB_ERR_STATE, "lb_lp_calibrate: no enabled network");
    if (m < 1 || m > 30) return fail(h, LB_ERR_ARG, "lb_lp_calibrate: restart length must be in 1..30");
    cudaSetDevice(h->device);
    int rc = ensure_krylov(h, m, true);
    if (rc) return rc;
    const int G = h->G;
    const size_t n = h->kry_n;
    mg_prepare(h);
    for (int g = 0; g < G; ++g) {
        if ((rc = mg_group_setup(h, g))) return rc;
        double* phi = h->d_phi_all + (size_t)g * n;
        // learned FGMRES from the first-flight moments (its answer is discarded) ...
        k_copy(h, phi, h->d_b, n);
        KrylovResult kl = moment_solve(h, h->d_b, phi, LB_SOLVER_FGMRES_ML, m, rtol, 0.0, 0, mg_table(h, g, g));
        if (kl.status) return kl.status;
        // ... then plain GMRES, whose answer feeds the groups below
        k_copy(h, phi, h->d_b, n);
        KrylovResult kp = moment_solve(h, h->d_b, phi, LB_SOLVER_GMRES, m, rtol, 0.0, 0, mg_table(h, g, g));
        if (kp.status) return kp.status;
        if (plain_iters) plain_iters[g] = kp.nmv;
        if (learned_iters) learned_iters[g] = kl.nmv;
    }
    cudaError_t e = cudaStreamSynchronize(h->stream);
    return e == cudaSuccess ? moments_tc_status(h) : cuda_fail(h, e, "lb_lp_calibrate");
}

int lb_mg_get_results(lb_handle* h, double* flux, double* dose) {
    if (!h || h->device < 0 || !h->d_dose) return LB_ERR_STATE;
    cudaSetDevice(h->device);
    cudaError_t e = cudaSuccess;
    if (flux) e = cudaMemcpyAsync(flux, h->d_flux, sizeof(double) * (size_t)h->G * h->NENK, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess && dose)
        e = cudaMemcpyAsync(dose, h->d_dose, sizeof(double) * (size_t)h->NENK, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    return e == cudaSuccess ? LB_OK : cuda_fail(h, e, "read results");
}


int lb_lp_generate(lb_handle* h, int samples_per_group, int iters, unsigned long long seed, long long* total) {
    if (!h || h->device < 0 || h->G < 1 || !h->d_phi_all)
        return h ? fail(h, LB_ERR_STATE, "lb_lp_generate: multigroup problem not set") : LB_ERR_ARG;
    if (samples_per_group < 0 || iters < 1) return fail(h, LB_ERR_ARG, "lb_lp_generate: bad arguments");
    cudaSetDevice(h->device);
    const int G = h->G, m = 30;
    int rc = ensure_krylov(h, m, false);
    if (rc) return rc;
    const size_t n = h->kry_n;
    mg_prepare(h);
    double* r = h->d_V;          // residual of the iterate
    double* err = h->d_V + n;    // its error
    for (int g = 0; g < G; ++g) {
        if ((rc = mg_group_setup(h, g))) return rc;
        // reference solution of the group (also the source of the groups below it)
        double* phi = h->d_phi_all + (size_t)g * n;
        k_copy(h, phi, h->d_b, n);
        const float* sigl = mg_table(h, g, g);
        DevOp mv = [h, sigl](const double* in, double* out) { return apply_A(h, in, out, sigl); };
        KrylovResult kr = gmres_device(h, n, h->d_b, phi, m, 1e-10, 0.0, 4000, mv, nullptr);
        if (kr.status) return kr.status;
        // source iteration from the first-flight moments: x_{k+1} = x_k + r_k, r_k = b - A x_k = A e_k
        double* x = h->d_x;
        k_copy(h, x, h->d_b, n);
        for (int k = 0; k < iters; ++k) {
            if ((rc = apply_A(h, x, r, sigl))) return rc;
            k_axpby(h, r, h->d_b, 1.0, -1.0, n);
            k_copy(h, err, phi, n);
            k_axpby(h, err, x, -1.0, 1.0, n);
            const long long cnt = samples_per_group / iters + (k < samples_per_group % iters ? 1 : 0);
            const unsigned long long sd = seed ^ (0x9E3779B97F4A7C15ull * (unsigned long long)(g * 1024 + k + 1));
            if ((rc = mlp_sample(h, r, err, cnt, sd))) return rc;
            k_axpby(h, x, r, 1.0, 1.0, n);
        }
    }
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "lb_lp_generate");
    if ((rc = moments_tc_status(h))) return rc;
    if (total) lb_lp_num_samples(h, total);
    return LB_OK;
}

}  // extern "C"
