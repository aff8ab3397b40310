// Batched dose solves: many independent multigroup problems -- each with its own mesh, quadrature,
// cross sections and beam -- advanced together on one GPU.
//
// The reference solves one problem per process (Main.f90:326-476).  Here every problem keeps its
// own handle (mesh, schedule, moment operators, Krylov workspace) and the batch drives them in
// lock step:
//   * groups: step g solves group g of every problem that has one;
//   * GMRES(m): all problems of the step run the same Arnoldi step at the same time; converged
//     problems drop out through a device-side activity mask;
//   * the matrix-vector product of a step (moment-to-discrete of every problem, ONE persistent
//     sweep launch over all (problem, direction) pairs, discrete-to-moment of every problem) is
//     captured once per group step as a CUDA graph and replayed for every Arnoldi step, on fixed
//     per-problem ping-pong buffers;
//   * the Gram-Schmidt dots, axpys and norms are segmented kernels: one launch for all problems.
// The sweep launch shape (threads per CTA) is chosen by timing the candidates on the batch.
#include "lb_internal.h"
#include "gmres_host.h"
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>

using namespace lb;

struct lb_handle : public lb::Handle {};

struct lb_batch {
    int device = 0;
    lb_handle* aux = nullptr;                  // owns the batch stream, reduction buffers, staging
    std::vector<lb_handle*> probs;
    std::vector<cudaStream_t> own_streams;     // each problem's own stream, restored on destroy
    std::vector<double*> wa, wb;               // per-problem Arnoldi ping-pong buffers
    std::vector<size_t> wlen;
    int* d_active = nullptr;                   // [cap] activity mask read by the kernels
    int* h_active = nullptr;                   // pinned mirror copied by the graphs
    int cap = 0;
    BatchWork* d_work = nullptr;
    int work_cap = 0;
    int nwork = 0;
    int* d_counter = nullptr;
    int sweep_threads = 0;                     // chosen by timing (0: not yet)
    float tune_ms[2] = {0.f, 0.f};
    cudaGraphExec_t gx[3] = {nullptr, nullptr, nullptr};   // residual, a->b, b->a
    cudaEvent_t ev[2] = {nullptr, nullptr};
    double last_ms = 0.0;
    long long graph_launches = 0, sweep_launches = 0;
    std::string err;
};

namespace {

int bfail(lb_batch* b, int code, const std::string& msg) {
    b->err = msg;
    return code;
}

int bcuda(lb_batch* b, cudaError_t e, const char* what) {
    return bfail(b, e == cudaErrorMemoryAllocation ? LB_ERR_OOM : LB_ERR_CUDA,
                 std::string(what) + ": " + cudaGetErrorString(e));
}

cudaStream_t bstream(lb_batch* b) { return b->aux->stream; }

void free_graphs(lb_batch* b) {
    for (auto& g : b->gx)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
}

int prop_error(lb_batch* b, lb_handle* h, int rc, int p) {
    char buf[64];
    std::snprintf(buf, sizeof buf, "problem %d: ", p);
    return bfail(b, rc, buf + (h ? h->err : std::string("error")));
}

// Work list of the batched sweep for the problems in `ids`, longest direction first.
int build_work(lb_batch* b, const std::vector<int>& ids, int threads) {
    std::vector<BatchWork> w;
    std::vector<double> cost;
    for (int p : ids) {
        lb_handle* h = b->probs[p];
        for (int i = 0; i < h->NI; ++i) {
            BatchWork x{};
            x.items = h->d_items + (size_t)i * h->NE;
            x.lvl_start = h->d_lvl_start + h->lvl_base[i];
            x.geom = h->d_geom;
            x.sigt = h->d_sigt;
            x.psi = h->d_psi + (size_t)i * (size_t)h->NENK;
            x.dir = make_float4((float)h->k[3 * i], (float)h->k[3 * i + 1], (float)h->k[3 * i + 2], (float)h->w[i]);
            x.nlev = h->nlev[i];
            x.Nm = h->Nm;
            x.problem = p;
            double c = 0.0;
            if (h->nclusters > 0) {
                // block schedule: block levels, one thread per block of kClusterSize elements
                x.crec = h->d_crec + h->crec_base_h[i];
                x.blk_elem = h->d_blk_elem;
                x.cl_start = h->d_cl_start + h->cl_base_h[i];
                x.ncl = h->ncl_h[i];
                if (h->ngeom > 0) {
                    x.ngeom = h->ngeom;
                    x.rec = h->d_rec;
                    x.gtab = h->d_gtab;
                    x.tmat = h->d_tmat;
                }
                const int* st = &h->cl_start_h[h->cl_base_h[i]];
                for (int L = 0; L < x.ncl; ++L) c += 1.0 + kClusterSize * std::ceil((double)(st[L + 1] - st[L]) / threads);
            } else {
                for (int L = 0; L < h->nlev[i]; ++L) {
                    const int sz = h->lvl_start[h->lvl_base[i] + L + 1] - h->lvl_start[h->lvl_base[i] + L];
                    c += 1.0 + std::ceil((double)sz / threads);
                }
            }
            w.push_back(x);
            cost.push_back(c);
        }
    }
    std::vector<int> ord(w.size());
    std::iota(ord.begin(), ord.end(), 0);
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int c) { return cost[a] > cost[c]; });
    std::vector<BatchWork> ws(w.size());
    for (size_t i = 0; i < ord.size(); ++i) ws[i] = w[ord[i]];
    if ((int)ws.size() > b->work_cap) {
        if (b->d_work) cudaFree(b->d_work);
        b->d_work = nullptr;
        b->work_cap = 0;
        cudaError_t e = cudaMalloc(&b->d_work, sizeof(BatchWork) * ws.size());
        if (e != cudaSuccess) return bcuda(b, e, "batch work list");
        b->work_cap = (int)ws.size();
    }
    cudaError_t e = cudaMemcpyAsync(b->d_work, ws.data(), sizeof(BatchWork) * ws.size(), cudaMemcpyHostToDevice,
                                    bstream(b));
    if (e == cudaSuccess) e = cudaStreamSynchronize(bstream(b));
    if (e != cudaSuccess) return bcuda(b, e, "batch work list");
    b->nwork = (int)ws.size();
    return LB_OK;
}

int sweep_all(lb_batch* b) {
    ++b->sweep_launches;
    int rc = launch_sweep_batch(bstream(b), b->d_work, b->nwork, b->d_counter, b->d_active, b->sweep_threads,
                                b->aux->sm_count);
    return rc ? bfail(b, rc, "batched sweep launch failed") : LB_OK;
}

// Times the sweep launch shapes on the current work list (contents of psi are overwritten later).
int tune_sweep(lb_batch* b, const std::vector<int>& ids) {
    const int cand[2] = {1024, 512};
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int c = 0; c < 2; ++c) {
        b->sweep_threads = cand[c];
        int rc = build_work(b, ids, cand[c]);
        if (!rc) rc = sweep_all(b);   // first launch loads the module
        cudaEventRecord(e0, bstream(b));
        if (!rc) rc = sweep_all(b);
        cudaEventRecord(e1, bstream(b));
        cudaError_t e = cudaEventSynchronize(e1);
        if (rc || e != cudaSuccess) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            return rc ? rc : bcuda(b, e, "sweep tuning");
        }
        cudaEventElapsedTime(&b->tune_ms[c], e0, e1);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->sweep_threads = b->tune_ms[1] < b->tune_ms[0] ? 512 : 1024;
    if (const char* v = std::getenv("LB_SWEEP_VERBOSE"))
        if (*v == '1')
            std::fprintf(stderr, "batched sweep: 1024 threads %.3f ms, 512 threads %.3f ms -> %d\n", b->tune_ms[0],
                         b->tune_ms[1], b->sweep_threads);
    return build_work(b, ids, b->sweep_threads);
}

// y_p = A x_p for every problem in ids (direct launches).  mode 0: y = x - D T^-1 M Sigma x
// (sigl = the group's within-group table); mode 1: y = D T^-1 M src (source of the group).
int matvec_launches(lb_batch* b, const std::vector<int>& ids, int g, int mode, const std::vector<const double*>& x,
                    const std::vector<double*>& y) {
    for (size_t q = 0; q < ids.size(); ++q) {
        lb_handle* h = b->probs[ids[q]];
        const int rc = mode == 0 ? launch_m2d(h, x[q], mg_table(h, g, g), nullptr, nullptr, h->d_psi)
                                 : launch_m2d(h, nullptr, nullptr, h->d_src, nullptr, h->d_psi);
        if (rc) return prop_error(b, h, rc, ids[q]);
    }
    int rc = sweep_all(b);
    if (rc) return rc;
    for (size_t q = 0; q < ids.size(); ++q) {
        lb_handle* h = b->probs[ids[q]];
        rc = mode == 0 ? launch_d2m(h, h->d_psi, x[q], 1.0, -1.0, y[q]) : launch_d2m(h, h->d_psi, nullptr, 0.0, 1.0, y[q]);
        if (rc) return prop_error(b, h, rc, ids[q]);
    }
    return LB_OK;
}

// Captures the mask upload + matvec of every problem in ids as one graph.
int capture(lb_batch* b, const std::vector<int>& ids, int g, const std::vector<const double*>& x,
            const std::vector<double*>& y, cudaGraphExec_t* out) {
    cudaStream_t s = bstream(b);
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return bcuda(b, e, "graph capture");
    e = cudaMemcpyAsync(b->d_active, b->h_active, sizeof(int) * b->probs.size(), cudaMemcpyHostToDevice, s);
    int rc = e == cudaSuccess ? matvec_launches(b, ids, g, 0, x, y) : LB_ERR_CUDA;
    cudaGraph_t graph = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(s, &graph);
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (e2 != cudaSuccess) return bcuda(b, e2, "graph capture");
    e = cudaGraphInstantiate(out, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return bcuda(b, e, "graph instantiate");
    return LB_OK;
}

int run_graph(lb_batch* b, cudaGraphExec_t g) {
    ++b->graph_launches;
    cudaError_t e = cudaGraphLaunch(g, bstream(b));
    return e == cudaSuccess ? LB_OK : bcuda(b, e, "graph launch");
}

struct PState {
    int p = 0;
    lb_handle* h = nullptr;
    size_t n = 0;
    double* x = nullptr;   // solution (group flux moments)
    GmresHost gh;
    std::vector<double> hh, h2, coef, G;   // G: Gram matrix V^T V of the cycle's basis, (m + 2)^2
    double fpar4 = 0.0, fpar5 = 0.0, hk = 0.0, hk2 = 0.0;
    int nmv = 0, status = LB_OK, kk = 0;
    bool done = false, brk = false, reorth = false, cont = false;
};

SegVec seg(double* w, const double* V, size_t ldv, size_t n) {
    SegVec s{};
    s.w = w;
    s.V = V;
    s.ldv = ldv;
    s.n2 = n / 2;
    s.scale = 1.0;
    return s;
}

int seg_grid(lb_batch* b) { return b->aux->sm_count * 4; }

// Lock-step restarted GMRES(m) for the problems `ids` at group g (SPARSKIT semantics per problem).
int batch_gmres(lb_batch* b, const std::vector<int>& ids, int g, int m, double rtol, double atol, int maxit,
                std::vector<int>& nmv_out, std::vector<int>& status_out) {
    Handle* ax = b->aux;
    const int P = (int)ids.size();
    std::vector<PState> st(P);
    for (int q = 0; q < P; ++q) {
        st[q].p = ids[q];
        st[q].h = b->probs[ids[q]];
        st[q].n = st[q].h->kry_n;
        st[q].x = st[q].h->d_phi_all + (size_t)g * st[q].n;
        st[q].gh.resize(m);
        st[q].hh.assign(m + 2, 0.0);
        st[q].h2.assign(m + 2, 0.0);
        st[q].G.assign((size_t)(m + 2) * (m + 2), 0.0);
    }
    // graphs of this group step: residual (x -> V0), a -> b, b -> a
    free_graphs(b);
    std::vector<const double*> xin(P), ain(P), bin(P);
    std::vector<double*> v0(P), aout(P), bout(P);
    for (int q = 0; q < P; ++q) {
        const int p = ids[q];
        xin[q] = st[q].x;
        v0[q] = st[q].h->d_V;
        ain[q] = b->wa[p];
        aout[q] = b->wb[p];
        bin[q] = b->wb[p];
        bout[q] = b->wa[p];
    }
    int rc;
    if ((rc = capture(b, ids, g, xin, v0, &b->gx[0]))) return rc;
    if ((rc = capture(b, ids, g, ain, aout, &b->gx[1]))) return rc;
    if ((rc = capture(b, ids, g, bin, bout, &b->gx[2]))) return rc;
    auto set_mask = [&](const std::vector<int>& which) {
        // the previous graph may still be reading the mask
        cudaStreamSynchronize(bstream(b));
        std::fill(b->h_active, b->h_active + b->probs.size(), 0);
        for (int q : which) b->h_active[st[q].p] = 1;
    };
    // |b| of every problem
    {
        std::vector<SegVec> sg;
        for (int q = 0; q < P; ++q) sg.push_back(seg(st[q].h->d_b, nullptr, 0, st[q].n));
        seg_assign_blocks(sg, seg_grid(b));
        std::vector<double> out;
        if ((rc = seg_dots_norm(ax, sg, 0, out))) return bfail(b, rc, ax->err);
        for (int q = 0; q < P; ++q) st[q].fpar4 = rtol * std::sqrt(out[q]) + atol;
    }
    std::vector<double> out;
    while (true) {
        std::vector<int> R;
        for (int q = 0; q < P; ++q)
            if (!st[q].done) R.push_back(q);
        if (R.empty()) break;
        // V0 = b - A x
        set_mask(R);
        if ((rc = run_graph(b, b->gx[0]))) return rc;
        {
            std::vector<SegVec> sg;
            for (int q : R) {
                SegVec s = seg(st[q].h->d_V, nullptr, 0, st[q].n);
                s.x = st[q].h->d_b;
                s.a = 1.0;
                s.b = -1.0;
                sg.push_back(s);
            }
            seg_assign_blocks(sg, seg_grid(b));
            if ((rc = seg_axpby_norm(ax, sg, out))) return bfail(b, rc, ax->err);
        }
        std::vector<int> A;
        std::vector<double> alpha_of(P, 0.0);
        for (size_t r = 0; r < R.size(); ++r) {
            PState& s = st[R[r]];
            ++s.nmv;
            const double alpha = std::sqrt(out[r]);
            if (std::isnan(alpha)) {
                s.status = LB_ERR_NAN;
                s.done = true;
                continue;
            }
            s.fpar5 = alpha;
            s.gh.start(alpha);
            s.G[0] = 1.0;
            if (alpha <= s.fpar4) {
                s.status = LB_OK;
                s.done = true;
                continue;
            }
            alpha_of[R[r]] = alpha;
            A.push_back(R[r]);
        }
        if (A.empty()) continue;
        {   // V0 /= alpha, copied into the a-buffer (input of the first Arnoldi product)
            std::vector<SegVec> sg;
            for (int q : A) {
                SegVec s = seg(st[q].h->d_V, nullptr, 0, st[q].n);
                s.scale = 1.0 / alpha_of[q];
                s.w2 = b->wa[st[q].p];
                sg.push_back(s);
            }
            seg_assign_blocks(sg, seg_grid(b));
            if ((rc = seg_axpy_scale(ax, sg, 0, {}))) return bfail(b, rc, ax->err);
        }
        int cur = 0;   // 0: current vector in a, product goes to b
        int k = 0;
        while (!A.empty()) {
            ++k;
            set_mask(A);
            if ((rc = run_graph(b, b->gx[1 + cur]))) return rc;
            std::vector<SegVec> sg;
            for (int q : A) {
                ++st[q].nmv;
                double* o = cur == 0 ? b->wb[st[q].p] : b->wa[st[q].p];
                sg.push_back(seg(o, st[q].h->d_V, st[q].n, st[q].n));
            }
            seg_assign_blocks(sg, seg_grid(b));
            // Gram-corrected classical Gram-Schmidt, as gmres_device: (1) projections and |w|^2;
            // G c = hh per problem; (2) w -= V c with h2 = V^T w and the exact |w|^2 in the same pass
            if ((rc = seg_dots_norm(ax, sg, k, out))) return bfail(b, rc, ax->err);
            const int ldg = m + 2;
            std::vector<double> coef;
            for (size_t a = 0; a < A.size(); ++a) {
                PState& s = st[A[a]];
                std::vector<double> hraw(out.begin() + a * (k + 1), out.begin() + a * (k + 1) + k);
                if (!gram_solve(s.G, ldg, k, hraw.data(), s.hh.data()))
                    for (int i = 0; i < k; ++i) s.hh[i] = hraw[i];
                coef.insert(coef.end(), s.hh.begin(), s.hh.begin() + k);
            }
            for (size_t a = 0; a < A.size(); ++a) sg[a].coef = (int)(a * k);
            if ((rc = seg_axpy_dots(ax, sg, k, coef, true, out))) return bfail(b, rc, ax->err);
            for (size_t a = 0; a < A.size(); ++a) {
                PState& s = st[A[a]];
                for (int i = 0; i < k; ++i) s.h2[i] = out[a * (k + 1) + i];
                s.hk2 = out[a * (k + 1) + k];
                s.reorth = false;
            }
            // (3) Hessenberg column, Givens rotation and the continue/leave decision
            std::vector<size_t> norm_re, norm_plain;
            for (size_t a = 0; a < A.size(); ++a) {
                PState& s = st[A[a]];
                s.hk = std::sqrt(std::max(0.0, s.hk2));
                s.brk = false;
                s.cont = false;
                if (std::isnan(s.hk)) {
                    s.status = LB_ERR_NAN;
                    s.done = true;
                    s.kk = -1;
                    continue;
                }
                if (!(s.hk > 0.0)) {
                    s.brk = true;
                    s.kk = k - 1;
                    continue;
                }
                const double alpha = s.gh.add_column(k, s.hh.data(), s.hk);
                s.fpar5 = alpha;
                s.kk = k;
                s.cont = k < m && !(alpha <= s.fpar4) && (maxit <= 0 || s.nmv < maxit);
                if (s.cont) {
                    norm_plain.push_back(a);
                    for (int i = 0; i < k; ++i)
                        s.G[(size_t)i * ldg + k] = s.G[(size_t)k * ldg + i] = s.h2[i] / s.hk;
                    s.G[(size_t)k * ldg + k] = 1.0;
                }
            }
            // normalise the continuing problems' new basis vector: v_k = w / hk, kept in the product
            // buffer (next input) and stored in V
            for (int pass = 0; pass < 2; ++pass) {
                const std::vector<size_t>& lst = pass == 0 ? norm_re : norm_plain;
                if (lst.empty()) continue;
                std::vector<SegVec> sn;
                std::vector<double> cn;
                for (size_t a : lst) {
                    PState& s = st[A[a]];
                    SegVec v = sg[a];
                    v.scale = 1.0 / s.hk;
                    v.w2 = s.h->d_V + (size_t)k * s.n;
                    v.coef = (int)cn.size();
                    if (pass == 0) cn.insert(cn.end(), s.h2.begin(), s.h2.begin() + k);
                    sn.push_back(v);
                }
                seg_assign_blocks(sn, seg_grid(b));
                if ((rc = seg_axpy_scale(ax, sn, pass == 0 ? k : 0, cn))) return bfail(b, rc, ax->err);
            }
            // problems leaving the cycle: back-substitution and x += V y, grouped by column count
            std::vector<int> next;
            std::vector<std::pair<int, size_t>> upd;   // (kept columns, index into A)
            for (size_t a = 0; a < A.size(); ++a) {
                PState& s = st[A[a]];
                if (s.done) continue;
                if (s.cont) {
                    next.push_back(A[a]);
                    continue;
                }
                const int kk = s.gh.solve(s.kk, s.coef);
                if (kk == 0) {
                    if (!s.brk) {
                        s.status = LB_ERR_BREAKDOWN;
                        s.done = true;
                    }
                    continue;
                }
                upd.push_back({kk, a});
            }
            std::sort(upd.begin(), upd.end());
            for (size_t i = 0; i < upd.size();) {
                size_t j = i;
                std::vector<SegVec> su;
                std::vector<double> cu;
                const int kk = upd[i].first;
                while (j < upd.size() && upd[j].first == kk) {
                    PState& s = st[A[upd[j].second]];
                    SegVec v = seg(s.x, s.h->d_V, s.n, s.n);
                    v.coef = (int)cu.size();
                    cu.insert(cu.end(), s.coef.begin(), s.coef.begin() + kk);
                    su.push_back(v);
                    ++j;
                }
                seg_assign_blocks(su, seg_grid(b));
                if ((rc = seg_axpy_scale(ax, su, kk, cu))) return bfail(b, rc, ax->err);
                i = j;
            }
            for (size_t a = 0; a < A.size(); ++a) {
                PState& s = st[A[a]];
                if (s.done || s.cont || s.brk) continue;   // breakdown: restart from the true residual
                if (s.fpar5 <= s.fpar4) {
                    s.status = LB_OK;
                    s.done = true;
                } else if (maxit > 0 && s.nmv >= maxit) {
                    s.status = LB_ERR_NOCONV;
                    s.done = true;
                }
            }
            A.swap(next);
            cur ^= 1;
        }
    }
    free_graphs(b);
    nmv_out.resize(P);
    status_out.resize(P);
    for (int q = 0; q < P; ++q) {
        nmv_out[q] = st[q].nmv;
        status_out[q] = st[q].status;
    }
    return LB_OK;
}

int ensure_batch_buffers(lb_batch* b, int m) {
    const int P = (int)b->probs.size();
    if (P > b->cap) {
        if (b->d_active) cudaFree(b->d_active);
        if (b->h_active) cudaFreeHost(b->h_active);
        b->d_active = nullptr;
        b->h_active = nullptr;
        cudaError_t e = cudaMalloc(&b->d_active, sizeof(int) * P);
        if (e == cudaSuccess) e = cudaMallocHost(&b->h_active, sizeof(int) * P);
        if (e != cudaSuccess) return bcuda(b, e, "batch masks");
        b->cap = P;
    }
    if (!b->d_counter) {
        cudaError_t e = cudaMalloc(&b->d_counter, sizeof(int));
        if (e != cudaSuccess) return bcuda(b, e, "batch counter");
    }
    b->wa.resize(P, nullptr);
    b->wb.resize(P, nullptr);
    b->wlen.resize(P, 0);
    for (int p = 0; p < P; ++p) {
        lb_handle* h = b->probs[p];
        int rc = ensure_krylov(h, m, false);
        if (rc) return prop_error(b, h, rc, p);
        if (b->wlen[p] != h->kry_n) {
            if (b->wa[p]) cudaFree(b->wa[p]);
            if (b->wb[p]) cudaFree(b->wb[p]);
            b->wa[p] = b->wb[p] = nullptr;
            cudaError_t e = cudaMalloc(&b->wa[p], sizeof(double) * h->kry_n);
            if (e == cudaSuccess) e = cudaMalloc(&b->wb[p], sizeof(double) * h->kry_n);
            if (e != cudaSuccess) return bcuda(b, e, "batch Arnoldi buffers");
            b->wlen[p] = h->kry_n;
        }
        h->d_active = b->d_active + p;
    }
    return LB_OK;
}

}  // namespace

extern "C" {

int lb_batch_create(int device, lb_batch** out) {
    if (!out) return LB_ERR_ARG;
    *out = nullptr;
    lb_batch* b = new lb_batch();
    b->device = device;
    int rc = lb_create(device, &b->aux);
    if (rc) {
        delete b;
        return rc;
    }
    b->aux->timing = false;
    *out = b;
    return LB_OK;
}

int lb_batch_destroy(lb_batch* b) {
    if (!b) return LB_ERR_ARG;
    cudaSetDevice(b->device);
    if (b->aux) cudaStreamSynchronize(b->aux->stream);
    free_graphs(b);
    for (size_t p = 0; p < b->probs.size(); ++p) {
        b->probs[p]->stream = b->own_streams[p];
        b->probs[p]->d_active = nullptr;
        lb_destroy(b->probs[p]);
    }
    for (double* v : b->wa)
        if (v) cudaFree(v);
    for (double* v : b->wb)
        if (v) cudaFree(v);
    if (b->d_active) cudaFree(b->d_active);
    if (b->h_active) cudaFreeHost(b->h_active);
    if (b->d_work) cudaFree(b->d_work);
    if (b->d_counter) cudaFree(b->d_counter);
    for (auto& e : b->ev)
        if (e) cudaEventDestroy(e);
    if (b->aux) lb_destroy(b->aux);
    delete b;
    return LB_OK;
}

int lb_batch_last_error(const lb_batch* b, char* buf, int len) {
    if (!b || !buf || len <= 0) return LB_ERR_ARG;
    std::snprintf(buf, (size_t)len, "%s", b->err.c_str());
    return LB_OK;
}

int lb_batch_add_problem(lb_batch* b, int NE, int NN, const double* rg, const int* node, const int* neighbors,
                         const int* mat, int Nm, int NI, const double* k, const double* w, int G, int Ls,
                         const double* sigt, const double* sigs, const double* dd, const double* unc,
                         const double* beam_dir, int* id) {
    if (!b) return LB_ERR_ARG;
    cudaSetDevice(b->device);
    lb_handle* h = nullptr;
    int rc = lb_create(b->device, &h);
    if (rc) return bfail(b, rc, "lb_batch_add_problem: cannot create a handle");
    if (!rc) rc = lb_set_mesh(h, NE, NN, rg, node, neighbors, mat, Nm);
    if (!rc) rc = lb_set_quadrature(h, NI, k, w);
    if (!rc) rc = lb_mg_set_problem(h, G, Ls, sigt, sigs, dd, unc, beam_dir);
    if (rc) {
        const int p = (int)b->probs.size();
        prop_error(b, h, rc, p);
        lb_destroy(h);
        return rc;
    }
    cudaStreamSynchronize(h->stream);
    b->own_streams.push_back(h->stream);
    h->stream = b->aux->stream;   // every launch of the batch goes to one stream (and its graphs)
    h->timing = false;
    b->probs.push_back(h);
    if (id) *id = (int)b->probs.size() - 1;
    return LB_OK;
}

int lb_batch_solve(lb_batch* b, int m, double rtol, double atol, int maxit, int* iters) {
    if (!b) return LB_ERR_ARG;
    if (b->probs.empty()) return bfail(b, LB_ERR_STATE, "lb_batch_solve: no problems");
    if (m < 1) m = 10;
    if (m > 30) return bfail(b, LB_ERR_ARG, "restart length must be <= 30");
    cudaSetDevice(b->device);
    const int P = (int)b->probs.size();
    int Gmax = 0;
    for (auto* h : b->probs) Gmax = std::max(Gmax, h->G);
    int rc = ensure_batch_buffers(b, m);
    if (rc) return rc;
    cudaStream_t s = bstream(b);
    if (!b->ev[0]) {
        cudaEventCreate(&b->ev[0]);
        cudaEventCreate(&b->ev[1]);
    }
    if (iters) std::fill(iters, iters + (size_t)P * Gmax, 0);
    for (auto* h : b->probs) {
        mg_prepare(h);
        cudaMemsetAsync(h->d_dose, 0, sizeof(double) * (size_t)h->NENK, s);
    }
    cudaEventRecord(b->ev[0], s);
    int first_err = LB_OK;
    for (int g = 0; g < Gmax; ++g) {
        std::vector<int> ids;
        for (int p = 0; p < P; ++p)
            if (b->probs[p]->G > g) ids.push_back(p);
        for (int p : ids)
            if ((rc = mg_group_sources(b->probs[p], g))) return prop_error(b, b->probs[p], rc, p);
        if (b->sweep_threads == 0) {
            std::fill(b->h_active, b->h_active + P, 1);
            cudaMemcpyAsync(b->d_active, b->h_active, sizeof(int) * P, cudaMemcpyHostToDevice, s);
            if ((rc = tune_sweep(b, ids))) return rc;
        } else if ((rc = build_work(b, ids, b->sweep_threads))) {
            return rc;
        }
        // b = D T^{-1} M src for every problem of the step, then x = b
        cudaStreamSynchronize(s);
        std::fill(b->h_active, b->h_active + P, 0);
        for (int p : ids) b->h_active[p] = 1;
        cudaMemcpyAsync(b->d_active, b->h_active, sizeof(int) * P, cudaMemcpyHostToDevice, s);
        std::vector<const double*> none(ids.size(), nullptr);
        std::vector<double*> bs;
        for (int p : ids) bs.push_back(b->probs[p]->d_b);
        if ((rc = matvec_launches(b, ids, g, 1, none, bs))) return rc;
        for (int p : ids) {
            lb_handle* h = b->probs[p];
            cudaMemcpyAsync(h->d_phi_all + (size_t)g * h->kry_n, h->d_b, sizeof(double) * h->kry_n,
                            cudaMemcpyDeviceToDevice, s);
        }
        std::vector<int> nmv, status;
        if ((rc = batch_gmres(b, ids, g, m, rtol, atol, maxit, nmv, status))) return rc;
        for (size_t q = 0; q < ids.size(); ++q) {
            const int p = ids[q];
            lb_handle* h = b->probs[p];
            if (iters) iters[(size_t)p * Gmax + g] = nmv[q];
            if (status[q] && !first_err) {
                first_err = status[q];
                char buf[96];
                std::snprintf(buf, sizeof buf, "problem %d group %d: Krylov status %d", p, g, status[q]);
                b->err = buf;
            }
            k_dose_tally(h, h->d_phi_all + (size_t)g * h->kry_n, h->d_unc, g == 0 ? 1.0 : 0.0,
                         h->d_dd + (size_t)g * h->Nm, h->d_mat, h->d_flux + (size_t)g * h->NENK, h->d_dose, h->NENK);
        }
    }
    cudaEventRecord(b->ev[1], s);
    cudaError_t e = cudaEventSynchronize(b->ev[1]);
    if (e != cudaSuccess) return bcuda(b, e, "batched solve");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]);
    b->last_ms = ms;
    for (int p = 0; p < P; ++p)
        if ((rc = moments_tc_status(b->probs[p]))) return prop_error(b, b->probs[p], rc, p);
    return first_err;
}

int lb_batch_get_results(lb_batch* b, int id, double* flux, double* dose) {
    if (!b || id < 0 || id >= (int)b->probs.size()) return LB_ERR_ARG;
    int rc = lb_mg_get_results(b->probs[id], flux, dose);
    return rc ? prop_error(b, b->probs[id], rc, id) : LB_OK;
}

int lb_batch_info(lb_batch* b, int* nproblems, int* max_groups, double* last_ms, int* sweep_threads,
                  long long* graph_launches, long long* sweep_launches) {
    if (!b) return LB_ERR_ARG;
    int Gmax = 0;
    for (auto* h : b->probs) Gmax = std::max(Gmax, h->G);
    if (nproblems) *nproblems = (int)b->probs.size();
    if (max_groups) *max_groups = Gmax;
    if (last_ms) *last_ms = b->last_ms;
    if (sweep_threads) *sweep_threads = b->sweep_threads;
    if (graph_launches) *graph_launches = b->graph_launches;
    if (sweep_launches) *sweep_launches = b->sweep_launches;
    return LB_OK;
}

}  // extern "C"
