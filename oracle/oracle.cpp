// ============================================================================================
//  Lionbolt transport-solve ORACLE  --  TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.
//
//  A CPU, FP64, OpenMP restatement of the reference Lionbolt (Fortran 2008) algorithms on the
//  within-group discrete-ordinates transport path.  Only the test-suite, the smoke check and the
//  CPU-baseline leg of the benchmark load this library; the CUDA product library never links,
//  calls or falls back to it.
//
//  Every function cites the reference file:line it restates (paths relative to the Lionbolt
//  repository root).  Array conventions: all indices are 0-based; a Fortran array A(i,j,...)
//  (column-major, 1-based) is stored here with identical memory order, i.e. A[...][j][i].
//
//  Parity pinning.  The reference cannot be compiled in this environment (pure Fortran, no
//  Fortran compiler, external NittanyPhysics dependency).  This restatement is therefore
//  pinned against (a) the discrete-ordinate tables printed in the reference's own run logs
//  (validation/photons_incident/water_tank_6MeV/lb.out:1739-2026 and
//  examples/three_beam_water_tank/lb.out), (b) the closed-form answers of the reference's
//  operator MMS drivers (validation/operators/ScatterMMS.f90:51-72, TransportMMS.f90:62-89).
//  Algorithms living in the absent NittanyPhysics v1.0.0 `core` library (Gauss-Legendre
//  nodes, Legendre polynomials, CROSS_PRODUCT/TRIPLE_PRODUCT, NORM2 as gfortran evaluates it)
//  are restated from their published definitions.
//
//  Compile with -ffp-contract=off so the FP64 face-orientation tests (k.n < -eps) are evaluated
//  without fused multiply-adds, as in the reference's DOT_PRODUCT.
// ============================================================================================
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdio>
#include <vector>
#include <algorithm>
#include <functional>
#include <omp.h>
#include <dlfcn.h>

namespace {

constexpr double PI = 3.14159265358979323846264338327950288;
constexpr double FOURPI = 4.0 * PI;
constexpr double TWOPI = 2.0 * PI;
constexpr double EPS64 = 2.220446049250313080847263336181640625e-16;   // EPSILON(1d0)

// gmsh local face -> local node map for linear tets, FiniteElementAnalysis.f90:129-132
constexpr int F2K[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};

// gfortran NORM2: scaled sum of squares (avoids overflow); result = scale*sqrt(ssq).
double norm2_scaled(const double* x, long n, long stride = 1) {
    double scale = 0.0, ssq = 1.0;
    for (long i = 0; i < n; ++i) {
        double v = x[i * stride];
        if (v != 0.0) {
            double a = std::fabs(v);
            if (scale < a) { double r = scale / a; ssq = 1.0 + ssq * r * r; scale = a; }
            else { double r = a / scale; ssq += r * r; }
        }
    }
    return scale * std::sqrt(ssq);
}

double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// CROSS_PRODUCT(a, b) = a x b (NittanyPhysics BasicMathFunctions, standard definition)
void cross3(const double* a, const double* b, double* c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

// Gauss-Legendre nodes/weights on [-1,1], ascending nodes (the order printed in lb.out).
// Restates NittanyPhysics PrepGaussLegendreQuadrature (called at SNPrep.f90:42 and
// FEAInnerProducts.f90:22) by Newton iteration on P_n.
void legendre_pair(int n, double z, double& pn, double& pnm1) {
    double p0 = 1.0, p1 = z;            // P_0, P_1
    for (int l = 2; l <= n; ++l) {
        double p2 = ((2.0 * l - 1.0) * z * p1 - (l - 1.0) * p0) / l;
        p0 = p1; p1 = p2;
    }
    pn = p1; pnm1 = p0;                  // valid for n >= 1
}

void gauss_legendre(int n, double* x, double* w) {
    for (int i = 0; i < n; ++i) {
        // i-th root counted from +1 (standard asymptotic guess), Newton-refined
        double z = std::cos(PI * (i + 0.75) / (n + 0.5));
        double pn, pnm1, dp;
        for (int it = 0; it < 100; ++it) {
            legendre_pair(n, z, pn, pnm1);
            dp = n * (z * pn - pnm1) / (z * z - 1.0);
            double dz = pn / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-16) break;
        }
        legendre_pair(n, z, pn, pnm1);
        dp = n * (z * pn - pnm1) / (z * z - 1.0);
        // root counted from the top -> ascending position n-1-i
        x[n - 1 - i] = z;
        w[n - 1 - i] = 2.0 / ((1.0 - z * z) * dp * dp);
    }
    // exact antisymmetry of nodes / symmetry of weights
    for (int i = 0; i < n / 2; ++i) {
        double a = 0.5 * (x[n - 1 - i] - x[i]);
        x[i] = -a; x[n - 1 - i] = a;
        double b = 0.5 * (w[i] + w[n - 1 - i]);
        w[i] = b; w[n - 1 - i] = b;
    }
    if (n % 2 == 1) x[n / 2] = 0.0;
}

// Legendre polynomials P_0..P_L at x (Bonnet recurrence); restates NittanyPhysics
// LegendrePolynomials (SNPrep.f90:117).
void legendre(int L, double x, double* P) {
    P[0] = 1.0;
    if (L >= 1) P[1] = x;
    for (int l = 2; l <= L; ++l) P[l] = ((2.0 * l - 1.0) * x * P[l - 1] - (l - 1.0) * P[l - 2]) / l;
}

// ------------------------------------------------------------------------------------------
// Literal 4x4 (of 8x8 scratch) LU with row pivoting, TransportAlgebra.f90:173-246
// ------------------------------------------------------------------------------------------
void local_lu(int n, double A[8][8], double b[8]) {   // A[row][col]
    double x[8];
    for (int k = 0; k < n - 1; ++k) {
        double maxval = std::fabs(A[k][k]);
        int pivot = k;
        for (int i = k + 1; i < n; ++i)
            if (std::fabs(A[i][k]) > maxval) { maxval = std::fabs(A[i][k]); pivot = i; }
        if (pivot != k) {
            for (int j = 0; j < 8; ++j) std::swap(A[k][j], A[pivot][j]);
            std::swap(b[k], b[pivot]);
        }
        for (int i = k + 1; i < n; ++i) {
            double factor = A[i][k] / A[k][k];
            A[i][k] = factor;
            for (int j = k + 1; j < n; ++j) A[i][j] = A[i][j] - factor * A[k][j];
            b[i] = b[i] - factor * b[k];
        }
    }
    x[n - 1] = b[n - 1] / A[n - 1][n - 1];
    for (int i = n - 2; i >= 0; --i) {
        x[i] = b[i];
        for (int j = i + 1; j < n; ++j) x[i] = x[i] - A[i][j] * x[j];
        x[i] = x[i] / A[i][i];
    }
    for (int i = 0; i < n; ++i) b[i] = x[i];
}

// Gauss-Jordan inverse with partial pivoting (stands in for dgetrf+dgetri,
// FiniteElementAnalysis.f90:171-180).  a is n x n row-major, inverted in place.
void invert(int n, double* a) {
    std::vector<double> m(n * 2 * n, 0.0);
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < n; ++j) m[i * 2 * n + j] = a[i * n + j];
        m[i * 2 * n + n + i] = 1.0;
    }
    for (int c = 0; c < n; ++c) {
        int p = c;
        for (int r = c + 1; r < n; ++r) if (std::fabs(m[r * 2 * n + c]) > std::fabs(m[p * 2 * n + c])) p = r;
        if (p != c) for (int j = 0; j < 2 * n; ++j) std::swap(m[c * 2 * n + j], m[p * 2 * n + j]);
        double d = m[c * 2 * n + c];
        for (int j = 0; j < 2 * n; ++j) m[c * 2 * n + j] /= d;
        for (int r = 0; r < n; ++r) {
            if (r == c) continue;
            double f = m[r * 2 * n + c];
            if (f == 0.0) continue;
            for (int j = 0; j < 2 * n; ++j) m[r * 2 * n + j] -= f * m[c * 2 * n + j];
        }
    }
    for (int i = 0; i < n; ++i) for (int j = 0; j < n; ++j) a[i * n + j] = m[i * 2 * n + n + j];
}

// ==========================================================================================
//  Oracle state: mesh + FEA (PostProcess.f90, FiniteElementAnalysis.f90), angular
//  (SNPrep.f90), sweep order (SweepOrder.f90, SweepArrays.f90), cross sections.
// ==========================================================================================
struct Oracle {
    // mesh
    int NE = 0, NN = 0, Nm = 1;
    std::vector<double> rg;      // [NN][3]
    std::vector<int> node;       // [NE][4]
    std::vector<int> nbr;        // [NE][4], -1 = boundary
    std::vector<int> mat;        // [NE]
    std::vector<double> nrm;     // [NE][4][3] outward unit normals
    std::vector<double> area;    // [NE][4]
    std::vector<double> vol;     // [NE]
    std::vector<double> detJ;    // [NE]
    std::vector<double> IC;      // [NE][3][4][4]  Fortran IC(k,kp,d,le) -> [le][d][kp][k]
    std::vector<double> IFM;     // [NE][4][4][4]  IFM(k,kp,f,le)      -> [le][f][kp][k]
    std::vector<double> IIM;     // [NE][4][4][4]
    long NENK = 0;
    // angular
    int NI = 0, L = 0;
    std::vector<double> k;       // [NI][3]
    std::vector<double> w;       // [NI]
    std::vector<double> YY;      // [L+1][NI][NI]   YY(ip,i,ell) -> [ell][i][ip]
    // schedule
    std::vector<int> sl;         // [NI][NE]   sl(es,i)
    std::vector<int> isl;        // [NI][NE]   isl(e,i)
    std::vector<uint8_t> isup;   // [NI][NE][4] IsUpstream
    std::vector<long> SAoffset;  // [NI][NE+1] (global offsets, as in the reference)
    std::vector<long> UFoffset;  // [NI][NE+1]
    std::vector<int> upfaces;    // [NZ]
    std::vector<long> ipsf;      // [NZ] 0-based start of the upstream element's block
    long NZ = 0;
    std::vector<int> nlevels;    // [NI]
    // physics
    std::vector<double> sigt;    // [Nm]
    std::vector<double> sigs;    // [Nm][L+1]   XS%s(ell,m) -> [m][ell]
    std::vector<double> YYS;     // [Nm][NI][NI] YYS(ip,i,m) -> [m][i][ip]
    bool have_xs = false;
    int nthreads = 0;
};

// ------------------------------------------------------------------------------------------
//  PostProcess.f90:45-102 (normals), :135-168 (areas), :243-279 (volumes)
// ------------------------------------------------------------------------------------------
void postprocess(Oracle& o) {
    const int NE = o.NE;
    o.nrm.assign((size_t)NE * 12, 0.0);
    o.area.assign((size_t)NE * 4, 0.0);
    o.vol.assign(NE, 0.0);
#pragma omp parallel for schedule(static)
    for (int e = 0; e < NE; ++e) {
        const int* nd = &o.node[(size_t)e * 4];
        double com[3] = {0, 0, 0};
        for (int kk = 0; kk < 4; ++kk) for (int d = 0; d < 3; ++d) com[d] += o.rg[(size_t)nd[kk] * 3 + d];
        for (int d = 0; d < 3; ++d) com[d] /= 4.0;
        for (int f = 0; f < 4; ++f) {
            // global face nodes are the sorted node triple (gmshprocessing.py:32-42, sort=True)
            int fn[3] = {nd[F2K[f][0]], nd[F2K[f][1]], nd[F2K[f][2]]};
            std::sort(fn, fn + 3);
            const double* r1p = &o.rg[(size_t)fn[0] * 3];
            const double* r2p = &o.rg[(size_t)fn[1] * 3];
            const double* r3p = &o.rg[(size_t)fn[2] * 3];
            double r1[3], r2[3], n[3];
            for (int d = 0; d < 3; ++d) { r1[d] = r2p[d] - r1p[d]; r2[d] = r3p[d] - r1p[d]; }
            cross3(r2, r1, n);                                   // n = CROSS_PRODUCT(r2, r1)
            double c[3];
            for (int d = 0; d < 3; ++d) c[d] = r1p[d] - com[d];
            double normfac = std::copysign(1.0, dot3(n, c)) / norm2_scaled(n, 3);
            for (int d = 0; d < 3; ++d) o.nrm[(size_t)e * 12 + f * 3 + d] = normfac * n[d];
            // face area, PostProcess.f90:141-146 (same sorted nodes)
            double cr[3];
            cross3(r2, r1, cr);
            o.area[(size_t)e * 4 + f] = 0.5 * norm2_scaled(cr, 3);
        }
        // volume: SIXTH*|TRIPLE_PRODUCT(r3,r2,r1)|, PostProcess.f90:271-277
        const double* p1 = &o.rg[(size_t)nd[0] * 3];
        double a1[3], a2[3], a3[3];
        for (int d = 0; d < 3; ++d) {
            a1[d] = o.rg[(size_t)nd[1] * 3 + d] - p1[d];
            a2[d] = o.rg[(size_t)nd[2] * 3 + d] - p1[d];
            a3[d] = o.rg[(size_t)nd[3] * 3 + d] - p1[d];
        }
        double cx[3];
        cross3(a2, a1, cx);
        o.vol[e] = std::fabs(dot3(a3, cx)) / 6.0;
    }
    o.NENK = (long)NE * 4;
}

// ------------------------------------------------------------------------------------------
//  FiniteElementAnalysis.f90:52-304 with FEAInnerProducts.f90:34-407 and Jacobians.f90:13-97.
//  Mass-eliminated IC, IFM, IIM for linear tets by 4-point Gauss-Legendre conical product.
// ------------------------------------------------------------------------------------------
void fea(Oracle& o) {
    const int Nq = 4;
    double xq[Nq], wq[Nq];
    gauss_legendre(Nq, xq, wq);
    auto tetsf = [](int kk, const double* r) { return kk == 0 ? 1.0 - (r[0] + r[1] + r[2]) : r[kk - 1]; };
    const double gradsf[4][3] = {{-1, -1, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    auto trisf = [](int kk, const double* r) { return kk == 0 ? 1.0 - (r[0] + r[1]) : r[kk - 1]; };
    // FEAMassRef (idx 4), FEAInnerProducts.f90:73-98
    double Mr[4][4] = {{0}}, ICr[4][4][3] = {{{0}}}, IFMr[3][3] = {{0}};
    for (int ii = 0; ii < Nq; ++ii) {
        double x = 0.5 * xq[ii] + 0.5;
        for (int j = 0; j < Nq; ++j) {
            double y = 0.5 * (1.0 - x) * xq[j] + 0.5 * (1.0 - x);
            for (int kk = 0; kk < Nq; ++kk) {
                double z = 0.5 * (1.0 - x - y) * xq[kk] + 0.5 * (1.0 - x - y);
                double r[3] = {x, y, z};
                double wt = wq[ii] * wq[j] * wq[kk] * 0.125 * (1.0 - x) * (1.0 - x - y);
                for (int kp = 0; kp < 4; ++kp) {
                    double ukp = tetsf(kp, r);
                    for (int k2 = 0; k2 < 4; ++k2) {
                        double uk = tetsf(k2, r);
                        Mr[k2][kp] += wt * uk * ukp;
                        for (int d = 0; d < 3; ++d) ICr[k2][kp][d] += wt * ukp * gradsf[k2][d];
                    }
                }
            }
        }
    }
    // FEAFaceMassRef (NK = 3), FEAInnerProducts.f90:263-283
    for (int ii = 0; ii < Nq; ++ii) {
        double x = 0.5 * xq[ii] + 0.5;
        for (int j = 0; j < Nq; ++j) {
            double y = 0.5 * (1.0 - x) * xq[j] + 0.5 * (1.0 - x);
            double r[2] = {x, y};
            for (int kp = 0; kp < 3; ++kp) {
                double ukp = trisf(kp, r);
                for (int k2 = 0; k2 < 3; ++k2) IFMr[k2][kp] += wq[ii] * wq[j] * 0.25 * (1.0 - x) * trisf(k2, r) * ukp;
            }
        }
    }
    double Minv[16];
    for (int a = 0; a < 4; ++a) for (int b = 0; b < 4; ++b) Minv[a * 4 + b] = Mr[a][b];
    invert(4, Minv);

    const int NE = o.NE;
    o.IC.assign((size_t)NE * 48, 0.0);
    o.IFM.assign((size_t)NE * 64, 0.0);
    o.IIM.assign((size_t)NE * 64, 0.0);
    o.detJ.assign(NE, 0.0);
#pragma omp parallel for schedule(static)
    for (int e = 0; e < NE; ++e) {
        const int* nd = &o.node[(size_t)e * 4];
        // Jacobian, Jacobians.f90:37-45,73-95: Jv(:,j) = r(node j+1) - r(node 1)
        double Jv[3][3];
        for (int j = 0; j < 3; ++j) for (int d = 0; d < 3; ++d)
            Jv[d][j] = o.rg[(size_t)nd[j + 1] * 3 + d] - o.rg[(size_t)nd[0] * 3 + d];
        double det = Jv[0][0] * (Jv[1][1] * Jv[2][2] - Jv[1][2] * Jv[2][1])
                   + Jv[0][1] * (Jv[1][2] * Jv[2][0] - Jv[1][0] * Jv[2][2])
                   + Jv[0][2] * (Jv[1][0] * Jv[2][1] - Jv[1][1] * Jv[2][0]);
        double A[3][3];
        A[0][0] = Jv[1][1] * Jv[2][2] - Jv[1][2] * Jv[2][1];
        A[0][1] = Jv[0][2] * Jv[2][1] - Jv[0][1] * Jv[2][2];
        A[0][2] = Jv[0][1] * Jv[1][2] - Jv[0][2] * Jv[1][1];
        A[1][0] = Jv[1][2] * Jv[2][0] - Jv[1][0] * Jv[2][2];
        A[1][1] = Jv[0][0] * Jv[2][2] - Jv[0][2] * Jv[2][0];
        A[1][2] = Jv[0][2] * Jv[1][0] - Jv[0][0] * Jv[1][2];
        A[2][0] = Jv[1][0] * Jv[2][1] - Jv[1][1] * Jv[2][0];
        A[2][1] = Jv[0][1] * Jv[2][0] - Jv[0][0] * Jv[2][1];
        A[2][2] = Jv[0][0] * Jv[1][1] - Jv[0][1] * Jv[1][0];
        double JiT[3][3];   // JvinvT = TRANSPOSE(A)/det
        for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) JiT[a][b] = A[b][a] / det;
        o.detJ[e] = det;
        double IM[4][4];
        for (int a = 0; a < 4; ++a) for (int b = 0; b < 4; ++b) IM[a][b] = Minv[a * 4 + b] / det;
        // MEFEAConvection, FEAInnerProducts.f90:311-338
        double ICt[4][4][3];
        for (int kp = 0; kp < 4; ++kp) for (int k2 = 0; k2 < 4; ++k2) for (int d = 0; d < 3; ++d) {
            double s = 0.0;
            for (int q = 0; q < 3; ++q) s += JiT[d][q] * ICr[k2][kp][q];
            ICt[k2][kp][d] = s;
        }
        for (int d = 0; d < 3; ++d) for (int k2 = 0; k2 < 4; ++k2) for (int kp = 0; kp < 4; ++kp) {
            double s = 0.0;
            for (int j = 0; j < 4; ++j) s += IM[k2][j] * ICt[j][kp][d];
            o.IC[(size_t)e * 48 + d * 16 + kp * 4 + k2] = det * s;
        }
        for (int f = 0; f < 4; ++f) {
            double normJs = 2.0 * o.area[(size_t)e * 4 + f];
            // MEFEAFaceMass, FEAInnerProducts.f90:340-371
            double F[4][4] = {{0}};
            for (int kp = 0; kp < 3; ++kp) for (int k2 = 0; k2 < 3; ++k2) F[F2K[f][k2]][F2K[f][kp]] = IFMr[k2][kp];
            for (int k2 = 0; k2 < 4; ++k2) for (int kp = 0; kp < 4; ++kp) {
                double s = 0.0;
                for (int j = 0; j < 4; ++j) s += IM[k2][j] * F[j][kp];
                o.IFM[(size_t)e * 64 + f * 16 + kp * 4 + k2] = s * normJs;
            }
            // MEFEAInterfaceMass, FEAInnerProducts.f90:373-407 (boundary faces keep zeros)
            int ep = o.nbr[(size_t)e * 4 + f];
            if (ep < 0) continue;
            const int* ndp = &o.node[(size_t)ep * 4];
            double G[4][4] = {{0}};
            for (int k2 = 0; k2 < 3; ++k2) {
                int k1 = F2K[f][k2];
                for (int kp = 0; kp < 3; ++kp) {
                    int kgp = nd[F2K[f][kp]];
                    int kk2 = -1;
                    for (int q = 0; q < 4; ++q) if (ndp[q] == kgp) { kk2 = q; break; }
                    if (kk2 >= 0) G[k1][kk2] = IFMr[k2][kp];
                }
            }
            for (int k2 = 0; k2 < 4; ++k2) for (int kp = 0; kp < 4; ++kp) {
                double s = 0.0;
                for (int j = 0; j < 4; ++j) s += IM[k2][j] * G[j][kp];
                o.IIM[(size_t)e * 64 + f * 16 + kp * 4 + k2] = s * normJs;
            }
        }
    }
}

// ------------------------------------------------------------------------------------------
//  SweepOrder.f90:105-207, literal: rescan every remaining element at every level.
// ------------------------------------------------------------------------------------------
int sweep_order_literal(Oracle& o) {
    const int NE = o.NE, NI = o.NI;
    o.sl.assign((size_t)NI * NE, -1);
    o.isl.assign((size_t)NI * NE, -1);
    o.isup.assign((size_t)NI * NE * 4, 0);
    o.nlevels.assign(NI, 0);
    int err = 0;
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < NI; ++i) {
        const double* kv = &o.k[(size_t)i * 3];
        std::vector<uint8_t> dep((size_t)NE * 4), rem(NE, 1);
        uint8_t* up = &o.isup[(size_t)i * NE * 4];
        for (int e = 0; e < NE; ++e)
            for (int f = 0; f < 4; ++f) {
                bool u = false;
                if (o.nbr[(size_t)e * 4 + f] >= 0) u = dot3(kv, &o.nrm[(size_t)e * 12 + f * 3]) < -EPS64;
                up[(size_t)e * 4 + f] = u;
                dep[(size_t)e * 4 + f] = u;
            }
        int* sli = &o.sl[(size_t)i * NE];
        int* isli = &o.isl[(size_t)i * NE];
        int es = 0, nlev = 0;
        while (true) {
            int lsss = 0;
            for (int e = 0; e < NE; ++e) {
                if (!rem[e]) continue;
                const uint8_t* d = &dep[(size_t)e * 4];
                if (!(d[0] | d[1] | d[2] | d[3])) {
                    sli[es] = e; isli[e] = es; rem[e] = 0; ++es; ++lsss;
                }
            }
            ++nlev;
            for (int esp = es - lsss; esp < es; ++esp) {
                int e = sli[esp];
                for (int f = 0; f < 4; ++f) {
                    int ep = o.nbr[(size_t)e * 4 + f];
                    if (ep < 0) continue;
                    int floc = -1;
                    for (int q = 0; q < 4; ++q) if (o.nbr[(size_t)ep * 4 + q] == e) { floc = q; break; }
                    if (floc >= 0) dep[(size_t)ep * 4 + floc] = 0;
                }
            }
            if (es == NE) break;
            if (lsss == 0) {
#pragma omp critical
                err = 1;
                break;
            }
        }
        o.nlevels[i] = nlev;
    }
    return err;
}

// Same level sets as sweep_order_literal, by per-level dependency counting (used for meshes too
// large for the literal O(levels*NE) rescan).  Each level is the ascending list of elements whose
// last pending upstream neighbour was released by the previous level.
int sweep_order_counting(Oracle& o) {
    const int NE = o.NE, NI = o.NI;
    o.sl.assign((size_t)NI * NE, -1);
    o.isl.assign((size_t)NI * NE, -1);
    o.isup.assign((size_t)NI * NE * 4, 0);
    o.nlevels.assign(NI, 0);
    int err = 0;
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < NI; ++i) {
        const double* kv = &o.k[(size_t)i * 3];
        uint8_t* up = &o.isup[(size_t)i * NE * 4];
        std::vector<int> cnt(NE, 0);
        std::vector<int> cur, nxt;
        for (int e = 0; e < NE; ++e) {
            for (int f = 0; f < 4; ++f) {
                bool u = false;
                if (o.nbr[(size_t)e * 4 + f] >= 0) u = dot3(kv, &o.nrm[(size_t)e * 12 + f * 3]) < -EPS64;
                up[(size_t)e * 4 + f] = u;
                cnt[e] += u;
            }
            if (cnt[e] == 0) cur.push_back(e);
        }
        int* sli = &o.sl[(size_t)i * NE];
        int* isli = &o.isl[(size_t)i * NE];
        int es = 0, nlev = 0;
        while (!cur.empty()) {
            for (int e : cur) { sli[es] = e; isli[e] = es; ++es; }
            ++nlev;
            nxt.clear();
            for (int e : cur)
                for (int f = 0; f < 4; ++f) {
                    int ep = o.nbr[(size_t)e * 4 + f];
                    if (ep < 0) continue;
                    for (int q = 0; q < 4; ++q)
                        if (o.nbr[(size_t)ep * 4 + q] == e) {
                            if (up[(size_t)ep * 4 + q] && --cnt[ep] == 0) nxt.push_back(ep);
                            break;
                        }
                }
            std::sort(nxt.begin(), nxt.end());
            cur.swap(nxt);
        }
        o.nlevels[i] = nlev;
        if (es != NE) {
#pragma omp critical
            err = 1;
        }
    }
    return err;
}

// ------------------------------------------------------------------------------------------
//  SweepArrays.f90:34-92
// ------------------------------------------------------------------------------------------
void sweep_arrays(Oracle& o) {
    const int NE = o.NE, NI = o.NI;
    o.SAoffset.assign((size_t)NI * (NE + 1), 0);
    long j = 0;
    for (int i = 0; i < NI; ++i) {
        for (int es = 0; es < NE; ++es) { o.SAoffset[(size_t)i * (NE + 1) + es] = j; j += 4; }
        o.SAoffset[(size_t)i * (NE + 1) + NE] = j;
    }
    long NZ = 0;
    for (size_t q = 0; q < o.isup.size(); ++q) NZ += o.isup[q];
    o.NZ = NZ;
    o.UFoffset.assign((size_t)NI * (NE + 1), 0);
    o.upfaces.assign(NZ, 0);
    o.ipsf.assign(NZ, 0);
    long iupf = 0;
    j = 0;
    for (int i = 0; i < NI; ++i) {
        for (int es = 0; es < NE; ++es) {
            int e = o.sl[(size_t)i * NE + es];
            int nup = 0;
            for (int f = 0; f < 4; ++f) {
                if (!o.isup[((size_t)i * NE + e) * 4 + f]) continue;
                ++nup;
                o.upfaces[iupf] = f;
                int eup = o.nbr[(size_t)e * 4 + f];
                int esp = o.isl[(size_t)i * NE + eup];
                o.ipsf[iupf] = o.SAoffset[(size_t)i * (NE + 1) + esp];
                ++iupf;
            }
            o.UFoffset[(size_t)i * (NE + 1) + es] = j;
            j += nup;
        }
        o.UFoffset[(size_t)i * (NE + 1) + NE] = j;
    }
}

// ------------------------------------------------------------------------------------------
//  ApplyInvertedDiagonal, TransportAlgebra.f90:108-171
// ------------------------------------------------------------------------------------------
inline void apply_inverted_diagonal(const Oracle& o, int e, double attn, const double* kv, double tmp8[8]) {
    double Td[8][8];
    for (int a = 0; a < 4; ++a) for (int b = 0; b < 4; ++b) Td[a][b] = 0.0;
    for (int a = 0; a < 4; ++a) Td[a][a] = attn;
    const double* ic = &o.IC[(size_t)e * 48];
    for (int d = 0; d < 3; ++d)
        for (int kp = 0; kp < 4; ++kp) for (int k2 = 0; k2 < 4; ++k2)
            Td[k2][kp] = Td[k2][kp] - kv[d] * ic[d * 16 + kp * 4 + k2];
    for (int f = 0; f < 4; ++f) {
        double kdotn = dot3(kv, &o.nrm[(size_t)e * 12 + f * 3]);
        if (kdotn < 0.0) continue;
        const double* ifm = &o.IFM[(size_t)e * 64 + f * 16];
        for (int kp = 0; kp < 4; ++kp) for (int k2 = 0; k2 < 4; ++k2)
            Td[k2][kp] = Td[k2][kp] + kdotn * ifm[kp * 4 + k2];
    }
    local_lu(4, Td, tmp8);
}

// Sweep for one direction on a sweep-ordered vector block s (TransportAlgebra.f90:66-103).
// s points at the start of the whole vector; offsets are the reference's global offsets.
void sweep_direction(const Oracle& o, int i, double* s) {
    const int NE = o.NE;
    const double* lk = &o.k[(size_t)i * 3];
    const long* SAo = &o.SAoffset[(size_t)i * (NE + 1)];
    const long* UFo = &o.UFoffset[(size_t)i * (NE + 1)];
    for (int es = 0; es < NE; ++es) {
        int e = o.sl[(size_t)i * NE + es];
        int m = o.mat[e];
        long ips = SAo[es];
        long iaf0 = UFo[es];
        long nup = UFo[es + 1] - iaf0;
        for (long fup = 0; fup < nup; ++fup) {
            int f = o.upfaces[iaf0 + fup];
            long ipsf = o.ipsf[iaf0 + fup];
            double kdotn = dot3(lk, &o.nrm[(size_t)e * 12 + f * 3]);
            const double* iim = &o.IIM[(size_t)e * 64 + f * 16];
            for (int k2 = 0; k2 < 4; ++k2) {
                double mm = 0.0;
                for (int kp = 0; kp < 4; ++kp) mm += iim[kp * 4 + k2] * s[ipsf + kp];
                s[ips + k2] = s[ips + k2] + (-kdotn * mm);
            }
        }
        double tmp8[8];
        for (int k2 = 0; k2 < 4; ++k2) tmp8[k2] = s[ips + k2];
        apply_inverted_diagonal(o, e, o.sigt[m], lk, tmp8);
        for (int k2 = 0; k2 < 4; ++k2) s[ips + k2] = tmp8[k2];
    }
}

// EncodeSweep.f90:27-63 (encode: natural -> sweep order; decode: back)
void encode_sweep(const Oracle& o, bool encode, double* s, std::vector<double>& t) {
    const int NE = o.NE, NI = o.NI;
    const long NENK = o.NENK;
    t.resize((size_t)NENK * NI);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < NI; ++i) {
        long ios = (long)i * NENK;
        for (int es = 0; es < NE; ++es) {
            int e = o.sl[(size_t)i * NE + es];
            if (encode) {
                long os2 = o.SAoffset[(size_t)i * (NE + 1) + es];
                long os1 = 4L * e + ios;
                for (int k2 = 0; k2 < 4; ++k2) t[os2 + k2] = s[os1 + k2];
            } else {
                long os2 = 4L * es + ios;
                long os1 = o.SAoffset[(size_t)i * (NE + 1) + e];
                for (int k2 = 0; k2 < 4; ++k2) t[os1 + k2] = s[os2 + k2];
            }
        }
    }
    std::memcpy(s, t.data(), sizeof(double) * (size_t)NENK * NI);
}

// TransportOp%MatInv ('SWEEP'), TransportOperator.f90:101-147
void transport_inv(const Oracle& o, double* s) {
    std::vector<double> t;
    encode_sweep(o, true, s, t);
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < o.NI; ++i) sweep_direction(o, i, s);
    encode_sweep(o, false, s, t);
}

// ScatteringOp%Physics YYS, ScatteringOperator.f90:263-269
void build_yys(Oracle& o) {
    const int NI = o.NI, Nm = o.Nm, L = o.L;
    o.YYS.assign((size_t)Nm * NI * NI, 0.0);
    for (int m = 0; m < Nm; ++m)
        for (int ell = 0; ell <= L; ++ell) {
            double s = o.sigs[(size_t)m * (L + 1) + ell];
            const double* yy = &o.YY[(size_t)ell * NI * NI];
            double* y = &o.YYS[(size_t)m * NI * NI];
            for (size_t q = 0; q < (size_t)NI * NI; ++q) y[q] = y[q] + yy[q] * s;
        }
}

// ApplyScattering / SNMGXS, ScatteringAlgebra.f90:13-55.  Nm == 1: the dgemm('N','N') product
// xw(sd,i) = sum_ip x(sd,ip) YYS(ip,i); Nm > 1: the per-node dgemv('T') loop over mat2sd.
void scatter_apply(const Oracle& o, double* x) {
    const int NI = o.NI;
    const long NENK = o.NENK;
    std::vector<double> xw((size_t)NENK * NI);
    if (o.Nm == 1) {
        const double* Y = o.YYS.data();
#pragma omp parallel for schedule(static)
        for (long sd0 = 0; sd0 < NENK; sd0 += 64) {
            long sd1 = std::min(NENK, sd0 + 64);
            for (int i = 0; i < NI; ++i) {
                double acc[64];
                for (long sd = sd0; sd < sd1; ++sd) acc[sd - sd0] = 0.0;
                for (int ip = 0; ip < NI; ++ip) {
                    double y = Y[(size_t)i * NI + ip];
                    const double* xp = &x[(size_t)ip * NENK];
                    for (long sd = sd0; sd < sd1; ++sd) acc[sd - sd0] += xp[sd] * y;
                }
                for (long sd = sd0; sd < sd1; ++sd) xw[(size_t)i * NENK + sd] = acc[sd - sd0];
            }
        }
    } else {
#pragma omp parallel for schedule(static)
        for (long sd = 0; sd < NENK; ++sd) {
            int m = o.mat[sd / 4];      // mat2sd: node sd belongs to element sd/4 (PostProcess.f90:434-453)
            const double* Y = &o.YYS[(size_t)m * NI * NI];
            std::vector<double> xt(NI);
            for (int ip = 0; ip < NI; ++ip) xt[ip] = x[(size_t)ip * NENK + sd];
            for (int i = 0; i < NI; ++i) {
                double acc = 0.0;
                for (int ip = 0; ip < NI; ++ip) acc += Y[(size_t)i * NI + ip] * xt[ip];
                xw[(size_t)i * NENK + sd] = acc;
            }
        }
    }
    std::memcpy(x, xw.data(), sizeof(double) * xw.size());
}

// The per-node dgemv loop of SNMGXS (ScatteringAlgebra.f90:39-48) with a BLAS dgemv: for every node
// sd of [sd0, sd1): xtmp = x(sd, 1:NI) (stride NENK), ytmp = YYS(:,:,mat)^T xtmp
// (dgemv('T', NI, NI, 1, YYS(:,:,mat), NI, xtmp, 1, 0, ytmp, 1)), xw(sd, 1:NI) = ytmp; nodes outside the
// range are left unchanged.  The reference walks the nodes serially; here OpenMP threads take
// node ranges, each calling a single-threaded dgemv.
using cblas_dgemv_t = void (*)(int, int, int, int, double, const double*, int, const double*, int, double, double*, int);
cblas_dgemv_t g_dgemv = nullptr;
constexpr int kCblasColMajor = 102, kCblasTrans = 112;

void scatter_apply_dgemv(const Oracle& o, double* x, long sd0, long sd1) {
    const int NI = o.NI;
    const long NENK = o.NENK;
    const long n = sd1 - sd0;
    std::vector<double> xw((size_t)n * NI);
#pragma omp parallel
    {
        std::vector<double> xt(NI), yt(NI);
#pragma omp for schedule(static)
        for (long sd = sd0; sd < sd1; ++sd) {
            const double* Y = &o.YYS[(size_t)o.mat[sd / 4] * NI * NI];
            for (int ip = 0; ip < NI; ++ip) xt[ip] = x[(size_t)ip * NENK + sd];
            g_dgemv(kCblasColMajor, kCblasTrans, NI, NI, 1.0, Y, NI, xt.data(), 1, 0.0, yt.data(), 1);
            for (int i = 0; i < NI; ++i) xw[(size_t)(sd - sd0) * NI + i] = yt[i];
        }
    }
#pragma omp parallel for schedule(static)
    for (long sd = sd0; sd < sd1; ++sd)
        for (int i = 0; i < NI; ++i) x[(size_t)i * NENK + sd] = xw[(size_t)(sd - sd0) * NI + i];
}

// BoltzmannOp%MatVec with Tprecond, BoltzmannOperator.f90:76-102: x <- x - T^{-1} K x
void boltzmann_matvec(const Oracle& o, double* x) {
    size_t n = (size_t)o.NENK * o.NI;
    std::vector<double> xw(x, x + n);
    scatter_apply(o, x);
    transport_inv(o, x);
#pragma omp parallel for schedule(static)
    for (size_t q = 0; q < n; ++q) x[q] = xw[q] - x[q];
}

double dot(const double* a, const double* b, size_t n) {
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (size_t q = 0; q < n; ++q) s += a[q] * b[q];
    return s;
}

// ------------------------------------------------------------------------------------------
//  SPARSKIT givens, third_party/SPARSKIT/iters.f:3225-3262
// ------------------------------------------------------------------------------------------
void givens(double& x, double& y, double& c, double& s) {
    if (x == 0.0 && y == 0.0) { c = 1.0; s = 0.0; }
    else if (std::fabs(y) > std::fabs(x)) {
        double t = x / y; x = std::sqrt(1.0 + t * t); s = std::copysign(1.0 / x, y); c = t * s;
    } else if (std::fabs(y) <= std::fabs(x)) {
        double t = y / x; y = std::sqrt(1.0 + t * t); c = std::copysign(1.0 / y, x); s = t * c;
    } else { x = 0.0; y = 0.0; c = 1.0; s = 0.0; }
    x = std::fabs(x * y);
}

// SPARSKIT mgsro(.FALSE., ...), iters.f:3465-3587.  Orthogonalise V[ind] against V[0..ind-1].
int mgsro(std::vector<std::vector<double>>& V, int ind, size_t n, double* hh) {
    const double reorth = 0.98;
    double* v = V[ind].data();
    double nrm0 = dot(v, v, n);
    double thr = nrm0 * reorth;
    if (nrm0 <= 0.0) return -1;
    if (!(nrm0 > 0.0 && 1.0 / nrm0 > 0.0)) return -2;
    for (int i = 0; i < ind; ++i) {
        const double* vi = V[i].data();
        double fct = dot(v, vi, n);
        hh[i] = fct;
#pragma omp parallel for schedule(static)
        for (size_t q = 0; q < n; ++q) v[q] = v[q] - fct * vi[q];
        if (fct * fct > thr) {
            fct = dot(v, vi, n);
            hh[i] = hh[i] + fct;
#pragma omp parallel for schedule(static)
            for (size_t q = 0; q < n; ++q) v[q] = v[q] - fct * vi[q];
        }
        nrm0 = nrm0 - hh[i] * hh[i];
        if (nrm0 < 0.0) nrm0 = 0.0;
        thr = nrm0 * reorth;
    }
    double nrm1 = std::sqrt(dot(v, v, n));
    hh[ind] = nrm1;
    if (nrm1 <= 0.0) return -3;
    double fct = 1.0 / nrm1;
#pragma omp parallel for schedule(static)
    for (size_t q = 0; q < n; ++q) v[q] = v[q] * fct;
    return 0;
}

// ------------------------------------------------------------------------------------------
//  Restarted GMRES(m) / FGMRES(m) with SPARSKIT semantics: gmres iters.f:1901-2206, fgmres
//  iters.f:2511-2795, stopping test ipar(3)=2 (||r|| <= rtol*||rhs|| + atol), as configured by
//  GMRESWrapper (SPARSKIT.f90:20-181).  Written as a direct loop instead of reverse
//  communication; the arithmetic sequence per iteration is the reference's.
//  precond == nullptr -> GMRES; otherwise FGMRES with right preconditioner z = precond(v).
//  Returns 0 converged, -1 iteration limit, -3 breakdown.  iters = ipar(7) (matvec count).
// ------------------------------------------------------------------------------------------
using Apply = std::function<void(const double* in, double* out)>;
int gmres_sparskit(size_t n, const double* rhs, double* sol, int m, double rtol, double atol, int maxit,
                   const Apply& matvec, const Apply* precond, int* iters_out, double* resid_out,
                   std::vector<double>* history) {
    if (m <= 1) m = 15;
    std::vector<std::vector<double>> V(m + 1, std::vector<double>(n));
    std::vector<std::vector<double>> Z;
    if (precond) Z.assign(m, std::vector<double>(n));
    std::vector<std::vector<double>> H(m + 1, std::vector<double>(m + 2, 0.0));   // H[col][row]
    std::vector<double> c(m + 1), s(m + 1), rs(m + 2);
    std::vector<double> tmp(n);
    int nmv = 0;
    double fpar4 = rtol * std::sqrt(dot(rhs, rhs, n)) + atol;
    double fpar5 = 0.0, fpar6 = 0.0;
    int status = 1;
    while (true) {
        // label 100/10: r = rhs - A sol
        matvec(sol, tmp.data());
        ++nmv;
        double* r = V[0].data();
#pragma omp parallel for schedule(static)
        for (size_t q = 0; q < n; ++q) r[q] = rhs[q] - tmp[q];
        double alpha = std::sqrt(dot(r, r, n));
        fpar5 = alpha;
        if (history) history->push_back(alpha);
        rs[1] = alpha;
        if (alpha <= fpar4) { status = 0; fpar6 = alpha; break; }
        double ia = 1.0 / alpha;
#pragma omp parallel for schedule(static)
        for (size_t q = 0; q < n; ++q) r[q] = ia * r[q];
        int k = 0;
        int ierr = 0;
        while (true) {
            ++k;
            const double* vin = V[k - 1].data();
            if (precond) { (*precond)(vin, Z[k - 1].data()); vin = Z[k - 1].data(); }
            matvec(vin, V[k].data());
            ++nmv;
            double hh[130];
            ierr = mgsro(V, k, n, hh);
            for (int i = 0; i <= k; ++i) H[k][i + 1] = hh[i];
            if (ierr == -3) { --k; break; }    // exact (lucky) breakdown: drop the null column, restart
            if (ierr < 0) break;
            for (int i = 1; i <= k - 1; ++i) {
                double a = H[k][i];
                double cc = c[i], ss = s[i];
                H[k][i] = cc * a + ss * H[k][i + 1];
                H[k][i + 1] = cc * H[k][i + 1] - ss * a;
            }
            double cc, ss;
            givens(H[k][k], H[k][k + 1], cc, ss);
            c[k] = cc; s[k] = ss;
            double a = -ss * rs[k];
            rs[k] = cc * rs[k];
            rs[k + 1] = a;
            alpha = std::fabs(a);
            fpar5 = alpha;
            if (history) history->push_back(alpha);
            if (k < m && !(alpha <= fpar4) && (maxit <= 0 || nmv < maxit)) continue;
            break;
        }
        // label 200: triangular solve (reduce k on a zero diagonal)
        while (k > 0 && H[k][k] == 0.0) --k;
        if (k == 0) { status = -3; break; }
        rs[k] = rs[k] / H[k][k];
        for (int i = k - 1; i >= 1; --i) {
            for (int ii = 1; ii <= i; ++ii) rs[ii] = rs[ii] - rs[i + 1] * H[i + 1][ii];
            rs[i] = rs[i] / H[i][i];
        }
        if (precond) {
            for (int i = 0; i < k; ++i) {
                const double* z = Z[i].data();
                double y = rs[i + 1];
#pragma omp parallel for schedule(static)
                for (size_t q = 0; q < n; ++q) sol[q] = sol[q] + y * z[q];
            }
        } else {
            double* wv = tmp.data();
            const double* v0 = V[0].data();
            double y0 = rs[1];
#pragma omp parallel for schedule(static)
            for (size_t q = 0; q < n; ++q) wv[q] = v0[q] * y0;
            for (int i = 1; i <= k - 1; ++i) {
                const double* vi = V[i].data();
                double y = rs[i + 1];
#pragma omp parallel for schedule(static)
                for (size_t q = 0; q < n; ++q) wv[q] = wv[q] + y * vi[q];
            }
#pragma omp parallel for schedule(static)
            for (size_t q = 0; q < n; ++q) sol[q] = sol[q] + wv[q];
        }
        fpar6 = fpar5;
        if (ierr != 0 && ierr != -3) { status = -3; break; }
        if (ierr == -3) { if (maxit > 0 && nmv >= maxit) { status = -1; break; } continue; }
        if ((nmv < maxit || maxit <= 0) && fpar6 > fpar4) continue;
        status = (fpar6 <= fpar4) ? 0 : -1;
        break;
    }
    if (iters_out) *iters_out = nmv;
    if (resid_out) *resid_out = (status == 0) ? fpar6 : fpar5;
    return status;
}

// real orthonormal spherical harmonics Y_lm, m = -l..l, index l*l + l + m
void real_sh(int Ls, const double* dir, double* Y) {
    double x = dir[0], y = dir[1], z = dir[2];
    double ct = z;
    double st = std::sqrt(std::max(0.0, 1.0 - z * z));
    double phi = std::atan2(y, x);
    std::vector<double> P((Ls + 1) * (Ls + 1), 0.0);   // P[l][m] associated Legendre (no Condon-Shortley)
    auto Pi = [&](int l, int mm) -> double& { return P[l * (Ls + 1) + mm]; };
    Pi(0, 0) = 1.0;
    for (int mm = 1; mm <= Ls; ++mm) Pi(mm, mm) = Pi(mm - 1, mm - 1) * (2.0 * mm - 1.0) * st;
    for (int mm = 0; mm < Ls; ++mm) Pi(mm + 1, mm) = (2.0 * mm + 1.0) * ct * Pi(mm, mm);
    for (int mm = 0; mm <= Ls; ++mm)
        for (int l = mm + 2; l <= Ls; ++l)
            Pi(l, mm) = ((2.0 * l - 1.0) * ct * Pi(l - 1, mm) - (l + mm - 1.0) * Pi(l - 2, mm)) / (l - mm);
    for (int l = 0; l <= Ls; ++l) {
        for (int mm = -l; mm <= l; ++mm) {
            int am = std::abs(mm);
            double ratio = 1.0;
            for (int q = l - am + 1; q <= l + am; ++q) ratio /= q;     // (l-|m|)!/(l+|m|)!
            double N = std::sqrt((2.0 * l + 1.0) / FOURPI * ratio);
            double v;
            if (mm == 0) v = N * Pi(l, 0);
            else if (mm > 0) v = std::sqrt(2.0) * N * Pi(l, am) * std::cos(am * phi);
            else v = std::sqrt(2.0) * N * Pi(l, am) * std::sin(am * phi);
            Y[l * l + l + mm] = v;
        }
    }
}

// ==========================================================================================
//  Moment-space restatement, for problems whose angular Krylov space does not fit in host
//  memory (768,000 tets x 288 directions: one FP64 angular vector is 7.08 GB and the reference's
//  GMRES workspace about 85 GB, with a 32-bit workspace size that overflows, SPARSKIT.f90:55-67).
//
//  The scattering kernel factorises exactly (Legendre addition theorem with real orthonormal
//  harmonics): YYS(i',i) = sum_l s_l w_i' (2l+1)/(4 pi) P_l(k_i.k_i') = sum_lm Y_lm(k_i) s_l w_i'
//  Y_lm(k_i'), i.e. K = M S D (ScatteringOperator.f90:263-269, ScatteringAlgebra.f90:13-55).  With
//  phi = D psi the fixed point (I - T^-1 K) psi = T^-1 q of BoltzmannOp%MatInv
//  (BoltzmannOperator.f90:106-151) becomes
//        A phi = (I - D T^-1 M S) phi = b = D T^-1 q,      psi = T^-1 (M S phi + q),
//  which GMRES/FGMRES (gmres_sparskit) solves on nm*NENK unknowns.  Angular vectors are never held
//  whole: every application streams the directions in batches (M for the batch, one literal sweep
//  per direction, D accumulated in ascending direction order), so the result does not depend on
//  the thread count.  The within-group loop of Main.f90:326-476 keeps the group moments in memory
//  instead of tapes.
// ==========================================================================================
struct MomentSpace {
    int Ls = 0, nm = 0;
    std::vector<double> Y;       // [NI][nm] Y_j(k_i)
    std::vector<int> lofj;       // [nm] Legendre order of moment j
    int batch = 16;              // directions per streamed batch
};

void moment_space_init(const Oracle& o, MomentSpace& ms, int Ls) {
    ms.Ls = Ls;
    ms.nm = (Ls + 1) * (Ls + 1);
    ms.Y.assign((size_t)o.NI * ms.nm, 0.0);
    for (int i = 0; i < o.NI; ++i) real_sh(Ls, &o.k[(size_t)i * 3], &ms.Y[(size_t)i * ms.nm]);
    ms.lofj.resize(ms.nm);
    for (int l = 0; l <= Ls; ++l)
        for (int j = l * l; j < (l + 1) * (l + 1); ++j) ms.lofj[j] = l;
    ms.batch = std::max(8, 2 * omp_get_max_threads());
}

// Sweep of direction i on a natural-order block psi[NENK] (psi[4e + k]): the arithmetic of
// sweep_direction (TransportAlgebra.f90:66-103) in the same order, with the upstream element's
// values read at 4*nbr instead of through the sweep-ordered offsets (EncodeSweep.f90 only moves
// values, so both give the same bits).  Upstream faces are visited in ascending local face order,
// the order SweepArrays.f90:34-92 stores them in.
void sweep_direction_natural(const Oracle& o, int i, double* psi) {
    const int NE = o.NE;
    const double* lk = &o.k[(size_t)i * 3];
    const int* sli = &o.sl[(size_t)i * NE];
    const uint8_t* up = &o.isup[(size_t)i * NE * 4];
    for (int es = 0; es < NE; ++es) {
        const int e = sli[es];
        double* pe = psi + 4L * e;
        for (int f = 0; f < 4; ++f) {
            if (!up[(size_t)e * 4 + f]) continue;
            const double* pu = psi + 4L * o.nbr[(size_t)e * 4 + f];
            double kdotn = dot3(lk, &o.nrm[(size_t)e * 12 + f * 3]);
            const double* iim = &o.IIM[(size_t)e * 64 + f * 16];
            for (int k2 = 0; k2 < 4; ++k2) {
                double mm = 0.0;
                for (int kp = 0; kp < 4; ++kp) mm += iim[kp * 4 + k2] * pu[kp];
                pe[k2] = pe[k2] + (-kdotn * mm);
            }
        }
        double tmp8[8];
        for (int k2 = 0; k2 < 4; ++k2) tmp8[k2] = pe[k2];
        apply_inverted_diagonal(o, e, o.sigt[o.mat[e]], lk, tmp8);
        for (int k2 = 0; k2 < 4; ++k2) pe[k2] = tmp8[k2];
    }
}

// y = D T^-1 (M s + q): s a moment source [nm][NENK] (or null), q an angular source [NI][NENK]
// (or null).  psi_out (optional) receives T^-1 (M s + q) [NI][NENK].
void moment_transport(const Oracle& o, const MomentSpace& ms, const double* s, const double* q, double* y,
                      double* psi_out) {
    const int NI = o.NI, nm = ms.nm, B = ms.batch;
    const long NENK = o.NENK;
    constexpr long CH = 512;
    std::vector<double> pb((size_t)B * NENK);
#pragma omp parallel for schedule(static)
    for (long q0 = 0; q0 < (long)nm * NENK; ++q0) y[q0] = 0.0;
    for (int i0 = 0; i0 < NI; i0 += B) {
        const int nb = std::min(B, NI - i0);
        // M for the batch
#pragma omp parallel for schedule(static)
        for (long c0 = 0; c0 < NENK; c0 += CH) {
            const long c1 = std::min(NENK, c0 + CH);
            for (int b = 0; b < nb; ++b) {
                double* __restrict__ p = &pb[(size_t)b * NENK];
                const double* Yi = &ms.Y[(size_t)(i0 + b) * nm];
                if (q) for (long sd = c0; sd < c1; ++sd) p[sd] = q[(size_t)(i0 + b) * NENK + sd];
                else for (long sd = c0; sd < c1; ++sd) p[sd] = 0.0;
                if (!s) continue;
                // p += sum_j Y_j s_j, accumulated in ascending j (four terms per pass over p)
                int j = 0;
                for (; j + 4 <= nm; j += 4) {
                    const double y0 = Yi[j], y1 = Yi[j + 1], y2 = Yi[j + 2], y3 = Yi[j + 3];
                    const double* __restrict__ s0 = s + (size_t)j * NENK;
                    const double* __restrict__ s1 = s0 + NENK;
                    const double* __restrict__ s2 = s1 + NENK;
                    const double* __restrict__ s3 = s2 + NENK;
                    for (long sd = c0; sd < c1; ++sd)
                        p[sd] = (((p[sd] + y0 * s0[sd]) + y1 * s1[sd]) + y2 * s2[sd]) + y3 * s3[sd];
                }
                for (; j < nm; ++j) {
                    const double yj = Yi[j];
                    const double* __restrict__ sj = s + (size_t)j * NENK;
                    for (long sd = c0; sd < c1; ++sd) p[sd] = p[sd] + yj * sj[sd];
                }
            }
        }
        // T^-1, one direction per thread
#pragma omp parallel for schedule(dynamic, 1)
        for (int b = 0; b < nb; ++b) sweep_direction_natural(o, i0 + b, &pb[(size_t)b * NENK]);
        if (psi_out) std::memcpy(psi_out + (size_t)i0 * NENK, pb.data(), sizeof(double) * (size_t)nb * NENK);
        // D, accumulated in ascending direction order
#pragma omp parallel for schedule(static)
        for (long c0 = 0; c0 < NENK; c0 += CH) {
            const long c1 = std::min(NENK, c0 + CH);
            for (int j = 0; j < nm; ++j) {
                double* __restrict__ yj = y + (size_t)j * NENK;
                auto cw = [&](int b) { return o.w[i0 + b] * ms.Y[(size_t)(i0 + b) * nm + j]; };
                // y_j += sum_b w_b Y_j(k_b) psi_b, accumulated in ascending direction order
                int b = 0;
                for (; b + 4 <= nb; b += 4) {
                    const double a0 = cw(b), a1 = cw(b + 1), a2 = cw(b + 2), a3 = cw(b + 3);
                    const double* __restrict__ p0 = &pb[(size_t)b * NENK];
                    const double* __restrict__ p1 = p0 + NENK;
                    const double* __restrict__ p2 = p1 + NENK;
                    const double* __restrict__ p3 = p2 + NENK;
                    for (long sd = c0; sd < c1; ++sd)
                        yj[sd] = (((yj[sd] + a0 * p0[sd]) + a1 * p1[sd]) + a2 * p2[sd]) + a3 * p3[sd];
                }
                for (; b < nb; ++b) {
                    const double a = cw(b);
                    const double* __restrict__ pp = &pb[(size_t)b * NENK];
                    for (long sd = c0; sd < c1; ++sd) yj[sd] = yj[sd] + a * pp[sd];
                }
            }
        }
    }
}

// s = S x: s[j][sd] = sigma_{l(j)}(mat(sd)) x[j][sd], sigl [Nm][Ls+1]
void moment_scale(const Oracle& o, const MomentSpace& ms, const double* sigl, const double* x, double* s) {
    const long NENK = o.NENK;
    const int nm = ms.nm, Ls = ms.Ls;
#pragma omp parallel for schedule(static)
    for (long sd = 0; sd < NENK; ++sd) {
        const double* sg = sigl + (size_t)o.mat[sd / 4] * (Ls + 1);
        for (int j = 0; j < nm; ++j) s[(size_t)j * NENK + sd] = sg[ms.lofj[j]] * x[(size_t)j * NENK + sd];
    }
}

// Right preconditioner of the pinned-FGMRES checks: z[j][sd] = d[j] v[j][sd].
void moment_diag_precond(const MomentSpace& ms, long NENK, const double* d, const double* v, double* z) {
#pragma omp parallel for schedule(static)
    for (long q = 0; q < (long)ms.nm * NENK; ++q) z[q] = d[q / NENK] * v[q];
}

}  // namespace

// ==========================================================================================
//  C entry points (ctypes)
// ==========================================================================================
extern "C" {

void or_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }
int or_get_threads(void) { return omp_get_max_threads(); }

void or_gauss_legendre(int n, double* x, double* w) { gauss_legendre(n, x, w); }

// SNPrep.f90:39-76.  Ng polar (Gauss-Legendre) x Nc azimuthal (Chebyshev); the reference uses
// Nc = 2*Ng (L = Ng-1).  Directions ordered j (azimuth) outer, i (polar) inner.
int or_sn_quadrature(int Ng, int Nc, double* k, double* w) {
    std::vector<double> mu(Ng), wG(Ng);
    gauss_legendre(Ng, mu.data(), wG.data());
    double wC = TWOPI / Nc;
    int ii = 0;
    for (int j = 1; j <= Nc; ++j) {
        double phi = (2 * j - 1) * PI / Nc;
        for (int i = 0; i < Ng; ++i) {
            double st = std::sqrt(1.0 - mu[i] * mu[i]);
            k[ii * 3 + 0] = std::cos(phi) * st;
            k[ii * 3 + 1] = std::sin(phi) * st;
            k[ii * 3 + 2] = mu[i];
            w[ii] = wG[i] * wC;
            ++ii;
        }
    }
    return ii;
}

// YY(ip,i,ell) = w(ip)*(2 ell+1) P_ell(k_i . k_ip)/(4 pi), SNPrep.f90:104-133.  Layout [ell][i][ip].
void or_yy(int NI, const double* k, const double* w, int L, double* YY) {
#pragma omp parallel for schedule(static)
    for (int ip = 0; ip < NI; ++ip) {
        std::vector<double> P(L + 1);
        for (int i = 0; i < NI; ++i) {
            double x = (i == ip) ? 1.0 : dot3(&k[i * 3], &k[ip * 3]);
            legendre(L, x, P.data());
            for (int ell = 0; ell <= L; ++ell) {
                double v = (i == ip) ? (2 * ell + 1) / FOURPI : (2 * ell + 1) * P[ell] / FOURPI;
                YY[((size_t)ell * NI + i) * NI + ip] = v * w[ip];
            }
        }
    }
}

void or_real_sh(int Ls, const double* dir, double* Y) { real_sh(Ls, dir, Y); }

void* or_create(int NE, int NN, const double* rg, const int* node, const int* nbr, const int* mat, int Nm) {
    Oracle* o = new Oracle();
    o->NE = NE; o->NN = NN; o->Nm = Nm;
    o->rg.assign(rg, rg + (size_t)NN * 3);
    o->node.assign(node, node + (size_t)NE * 4);
    o->nbr.assign(nbr, nbr + (size_t)NE * 4);
    o->mat.assign(mat, mat + NE);
    postprocess(*o);
    fea(*o);
    return o;
}

void or_destroy(void* h) { delete static_cast<Oracle*>(h); }

long or_nenk(void* h) { return static_cast<Oracle*>(h)->NENK; }

// normals [NE][4][3], areas [NE][4], volumes [NE], detJ [NE], IC [NE][3][4][4], IFM/IIM [NE][4][4][4]
void or_get_geometry(void* h, double* n, double* area, double* vol, double* detJ, double* IC, double* IFM, double* IIM) {
    Oracle* o = static_cast<Oracle*>(h);
    if (n) std::memcpy(n, o->nrm.data(), sizeof(double) * o->nrm.size());
    if (area) std::memcpy(area, o->area.data(), sizeof(double) * o->area.size());
    if (vol) std::memcpy(vol, o->vol.data(), sizeof(double) * o->vol.size());
    if (detJ) std::memcpy(detJ, o->detJ.data(), sizeof(double) * o->detJ.size());
    if (IC) std::memcpy(IC, o->IC.data(), sizeof(double) * o->IC.size());
    if (IFM) std::memcpy(IFM, o->IFM.data(), sizeof(double) * o->IFM.size());
    if (IIM) std::memcpy(IIM, o->IIM.data(), sizeof(double) * o->IIM.size());
}

// TransportOp%SpaceAngle: quadrature + BuildSpaceAngle (SweepOrder + SweepArrays) + YY.
// literal == 1 selects the reference's rescanning SweepOrder, 0 the counting builder, 2 builds no
// schedule (quadrature and YY only, for scattering-only use).
// Returns 0, or 4 (LB_ERR_CYCLE) when a level makes no progress (SweepOrder.f90:178-184).
int or_set_angular(void* h, int NI, const double* k, const double* w, int L, int literal) {
    Oracle* o = static_cast<Oracle*>(h);
    o->NI = NI; o->L = L;
    o->k.assign(k, k + (size_t)NI * 3);
    o->w.assign(w, w + NI);
    o->YY.assign((size_t)(L + 1) * NI * NI, 0.0);
    or_yy(NI, k, w, L, o->YY.data());
    o->have_xs = false;
    if (literal == 2) return 0;   // quadrature and YY only: enough for ScatteringOp
    int err = literal ? sweep_order_literal(*o) : sweep_order_counting(*o);
    if (err) return 4;
    sweep_arrays(*o);
    o->have_xs = false;
    return 0;
}

long or_nz(void* h) { return static_cast<Oracle*>(h)->NZ; }

// sl/isl [NI][NE]; SAoffset/UFoffset [NI][NE+1]; upfaces/ipsf [NZ]; nlevels [NI]
void or_get_schedule(void* h, int* sl, int* isl, long* SAoffset, long* UFoffset, int* upfaces, long* ipsf, int* nlevels) {
    Oracle* o = static_cast<Oracle*>(h);
    if (sl) std::memcpy(sl, o->sl.data(), sizeof(int) * o->sl.size());
    if (isl) std::memcpy(isl, o->isl.data(), sizeof(int) * o->isl.size());
    if (SAoffset) std::memcpy(SAoffset, o->SAoffset.data(), sizeof(long) * o->SAoffset.size());
    if (UFoffset) std::memcpy(UFoffset, o->UFoffset.data(), sizeof(long) * o->UFoffset.size());
    if (upfaces) std::memcpy(upfaces, o->upfaces.data(), sizeof(int) * o->upfaces.size());
    if (ipsf) std::memcpy(ipsf, o->ipsf.data(), sizeof(long) * o->ipsf.size());
    if (nlevels) std::memcpy(nlevels, o->nlevels.data(), sizeof(int) * o->nlevels.size());
}

// sigt [Nm], sigs [Nm][L+1] (XS%t, XS%s(0:L,m)); builds YYS
int or_set_xs(void* h, const double* sigt, const double* sigs) {
    Oracle* o = static_cast<Oracle*>(h);
    o->sigt.assign(sigt, sigt + o->Nm);
    o->sigs.assign(sigs, sigs + (size_t)o->Nm * (o->L + 1));
    build_yys(*o);
    o->have_xs = true;
    return 0;
}

int or_transport_inv(void* h, double* s) { transport_inv(*static_cast<Oracle*>(h), s); return 0; }

// Loads a CBLAS library (the OpenBLAS bundled with scipy) for or_scatter_apply_dgemv: its
// cblas_dgemv entry `dgemv_name`, and `threads_name` (optional) called with 1 so that every OpenMP
// thread runs a single-threaded dgemv.  Returns 0, or 1 when the library or symbol is missing.
int or_set_blas(const char* path, const char* dgemv_name, const char* threads_name) {
    void* lib = dlopen(path, RTLD_NOW | RTLD_LOCAL);
    if (!lib) return 1;
    g_dgemv = reinterpret_cast<cblas_dgemv_t>(dlsym(lib, dgemv_name));
    if (!g_dgemv) return 1;
    if (threads_name) {
        auto set_threads = reinterpret_cast<void (*)(int)>(dlsym(lib, threads_name));
        if (set_threads) set_threads(1);
    }
    return 0;
}

// K x through the reference's per-node dgemv path on nodes [sd0, sd1) (all nodes: 0, NENK).
int or_scatter_apply_dgemv(void* h, double* x, long sd0, long sd1) {
    Oracle* o = static_cast<Oracle*>(h);
    if (!g_dgemv) return 1;
    if (!o->have_xs || sd0 < 0 || sd1 > o->NENK || sd0 > sd1) return 2;
    scatter_apply_dgemv(*o, x, sd0, sd1);
    return 0;
}
int or_scatter_apply(void* h, double* x) { scatter_apply(*static_cast<Oracle*>(h), x); return 0; }
int or_boltzmann_matvec(void* h, double* x) { boltzmann_matvec(*static_cast<Oracle*>(h), x); return 0; }

// BoltzmannOp%MatInv, BoltzmannOperator.f90:106-151 (Tprecond = SN).
// solver 0 = SI (SourceIteration.f90:3-82), 1 = GMRES(m) (GMRESWrapper, guess s/sigt(1)).
// On return s holds the solution.  history (optional, length hist_len) receives residual norms.
int or_boltzmann_solve(void* h, double* s, int solver, int m, double rtol, double atol, int maxit,
                       int* iters, double* resid, double* history, int hist_len, int* hist_n) {
    Oracle* o = static_cast<Oracle*>(h);
    size_t n = (size_t)o->NENK * o->NI;
    transport_inv(*o, s);
    std::vector<double> hist;
    int status = 0;
    if (solver == 0) {
        std::vector<double> wv(s, s + n);
        double norms = norm2_scaled(s, (long)n);
        int it = 1;
        scatter_apply(*o, wv.data());
        transport_inv(*o, wv.data());
        for (size_t q = 0; q < n; ++q) s[q] = s[q] + wv[q];
        double rn = 0.0;
        while (true) {
            ++it;
            rn = norm2_scaled(wv.data(), (long)n);
            hist.push_back(rn);
            if (rn <= atol + norms * rtol) break;
            if (maxit > 0 && it > maxit) { status = -1; break; }
            scatter_apply(*o, wv.data());
            transport_inv(*o, wv.data());
            for (size_t q = 0; q < n; ++q) s[q] = s[q] + wv[q];
        }
        if (iters) *iters = it;
        if (resid) *resid = rn;
    } else {
        std::vector<double> rhs(s, s + n), xg(n);
        double st1 = o->sigt[0];
        for (size_t q = 0; q < n; ++q) xg[q] = s[q] / st1;
        Apply mv = [o, n](const double* in, double* out) {
            std::memcpy(out, in, sizeof(double) * n);
            boltzmann_matvec(*o, out);
        };
        status = gmres_sparskit(n, rhs.data(), xg.data(), m, rtol, atol, maxit, mv, nullptr, iters, resid, &hist);
        std::memcpy(s, xg.data(), sizeof(double) * n);
    }
    if (history && hist_n) {
        int c = std::min<int>(hist_len, (int)hist.size());
        for (int q = 0; q < c; ++q) history[q] = hist[q];
        *hist_n = (int)hist.size();
    }
    return status;
}

// Fluence, LinearOperatorClass.f90:154-174: fl(sd) = sum_i w(i) v((i-1)NENK + sd)
void or_fluence(void* h, const double* v, double* fl) {
    Oracle* o = static_cast<Oracle*>(h);
    const long NENK = o->NENK;
    for (long sd = 0; sd < NENK; ++sd) fl[sd] = 0.0;
    for (int i = 0; i < o->NI; ++i)
        for (long sd = 0; sd < NENK; ++sd) fl[sd] = fl[sd] + o->w[i] * v[(size_t)i * NENK + sd];
}

// ------------------------------------------------------------------------------------------
//  Multigroup driver, Main.f90:326-476 with PIEISource (Main.f90:584-671) and the dose tally
//  (CalculateDeposition Main.f90:750-824, TallyDeposition.f90:19), angular space, FP64.
//  Beam: a monodirectional uncollided flux psi_unc(r, Omega) = delta(Omega - Omega_b) u(r) in
//  group 0 only (the host-built synthetic first-collision data; the reference ray-traces it in
//  FCSSource.f90/AddAngularFluence.f90).  K applied to it is the closed form
//  sum_l sigma_l (2l+1)/(4 pi) P_l(k_i . Omega_b) u(r).
//    G groups; sigt [G][Nm]; sigs [G'][G][Nm][L+1] transfer g'->g; dd [G][Nm];
//    unc [NENK] (u at every DG node), beam_dir [3].
//  Outputs: flux [G][NENK] (scalar fluence incl. uncollided), dose [NENK].
//  solver 0 SI / 1 GMRES(m).  iters_out [G].
// ------------------------------------------------------------------------------------------
int or_multigroup(void* h, int G, const double* sigt, const double* sigs, const double* dd, const double* unc,
                  const double* beam_dir, int solver, int m, double rtol, double atol, int maxit,
                  double* flux, double* dose, int* iters_out) {
    Oracle* o = static_cast<Oracle*>(h);
    const int NI = o->NI, Nm = o->Nm, L = o->L;
    const long NENK = o->NENK;
    size_t n = (size_t)NENK * NI;
    std::vector<std::vector<double>> psi(G);     // tapes: collided angular flux per group
    std::vector<double> s(n), w1(n);
    // beam angular factor per (direction, ell)
    std::vector<double> Pb((size_t)NI * (L + 1));
    for (int i = 0; i < NI; ++i) legendre(L, dot3(&o->k[i * 3], beam_dir), &Pb[(size_t)i * (L + 1)]);
    for (long sd = 0; sd < NENK; ++sd) dose[sd] = 0.0;
    for (int g = 0; g < G; ++g) {
        std::fill(s.begin(), s.end(), 0.0);
        // EI: sum_{g'<g} K_{g'->g} psi_{g'}   (Main.f90:584-629)
        for (int gp = 0; gp < g; ++gp) {
            o->sigt.assign(sigt + (size_t)gp * Nm, sigt + (size_t)(gp + 1) * Nm);
            o->sigs.assign(sigs + ((size_t)gp * G + g) * Nm * (L + 1), sigs + ((size_t)gp * G + g + 1) * Nm * (L + 1));
            bool allzero = true;
            for (double v : o->sigs) if (v != 0.0) allzero = false;
            if (allzero) continue;
            build_yys(*o);
            w1 = psi[gp];
            scatter_apply(*o, w1.data());
            for (size_t q = 0; q < n; ++q) s[q] = s[q] + w1[q];
        }
        // first-collision source of the group-0 uncollided flux into group g
        {
            const double* sg = sigs + ((size_t)0 * G + g) * Nm * (L + 1);
#pragma omp parallel for schedule(static)
            for (int i = 0; i < NI; ++i)
                for (long sd = 0; sd < NENK; ++sd) {
                    int mm = o->mat[sd / 4];
                    double a = 0.0;
                    for (int ell = 0; ell <= L; ++ell)
                        a += sg[(size_t)mm * (L + 1) + ell] * (2 * ell + 1) / FOURPI * Pb[(size_t)i * (L + 1) + ell];
                    s[(size_t)i * NENK + sd] += a * unc[sd];
                }
        }
        // within-group operator for group g
        o->sigt.assign(sigt + (size_t)g * Nm, sigt + (size_t)(g + 1) * Nm);
        o->sigs.assign(sigs + ((size_t)g * G + g) * Nm * (L + 1), sigs + ((size_t)g * G + g + 1) * Nm * (L + 1));
        build_yys(*o);
        int it = 0;
        double res = 0.0;
        int st = or_boltzmann_solve(o, s.data(), solver, m, rtol, atol, maxit, &it, &res, nullptr, 0, nullptr);
        if (iters_out) iters_out[g] = it;
        if (st != 0) return 6;
        psi[g] = s;
        // fluence and dose (uncollided added for group 0)
        double* fl = flux + (size_t)g * NENK;
        or_fluence(o, s.data(), fl);
        if (g == 0) for (long sd = 0; sd < NENK; ++sd) fl[sd] += unc[sd];
        for (long sd = 0; sd < NENK; ++sd) dose[sd] += dd[(size_t)g * Nm + o->mat[sd / 4]] * fl[sd];
        if (g == 0) {
            // tape holds collided + uncollided (Main.f90:443); the uncollided part's downscatter
            // is applied in closed form above, so only the collided flux is stored here.
        }
    }
    return 0;
}


// ------------------------------------------------------------------------------------------
//  Moment-space entry points (see MomentSpace above).
// ------------------------------------------------------------------------------------------

// TransportOp%SpaceAngle for the moment-space path: the level sets of SweepOrder.f90 (counting
// builder: sl, isl, IsUpstream) without the sweep-ordered offset arrays or YY, which the streamed
// sweeps do not use.  Returns 0, or 4 (LB_ERR_CYCLE) when a level makes no progress.
int or_set_angular_streamed(void* h, int NI, const double* k, const double* w) {
    Oracle* o = static_cast<Oracle*>(h);
    o->NI = NI;
    o->L = 0;
    o->k.assign(k, k + (size_t)NI * 3);
    o->w.assign(w, w + NI);
    o->YY.clear();
    o->SAoffset.clear(); o->UFoffset.clear(); o->upfaces.clear(); o->ipsf.clear();
    int err = sweep_order_counting(*o);
    long NZ = 0;
    for (size_t q = 0; q < o->isup.size(); ++q) NZ += o->isup[q];
    o->NZ = NZ;
    o->have_xs = false;
    return err ? 4 : 0;
}

// Total cross sections sigt[Nm] of the sweeps (TransportOp%Physics, XS%t).
int or_set_sigt(void* h, const double* sigt) {
    Oracle* o = static_cast<Oracle*>(h);
    o->sigt.assign(sigt, sigt + o->Nm);
    return 0;
}

// y[nm][NENK] = D T^-1 (M s + q) with s [nm][NENK] and q [NI][NENK] (either may be null);
// psi (optional) receives T^-1 (M s + q).
int or_moment_transport(void* h, int Ls, const double* s, const double* q, double* y, double* psi) {
    Oracle* o = static_cast<Oracle*>(h);
    if (o->sigt.empty() || o->sl.empty()) return 8;
    MomentSpace ms;
    moment_space_init(*o, ms, Ls);
    moment_transport(*o, ms, s, q, y, psi);
    return 0;
}

namespace {
// A phi = phi - D T^-1 M S phi as a gmres_sparskit operator (scratch: one moment vector).
Apply moment_operator(const Oracle& o, const MomentSpace& ms, const double* sigl, std::vector<double>& scratch) {
    const size_t n = (size_t)ms.nm * o.NENK;
    scratch.resize(n);
    return [&o, &ms, sigl, &scratch, n](const double* in, double* out) {
        moment_scale(o, ms, sigl, in, scratch.data());
        moment_transport(o, ms, scratch.data(), nullptr, out, nullptr);
#pragma omp parallel for schedule(static)
        for (size_t q = 0; q < n; ++q) out[q] = in[q] - out[q];
    };
}
}  // namespace

// y = A x = x - D T^-1 M S x, sigl [Nm][Ls+1] the within-group scattering moments XS%s(l, m).
int or_moment_apply(void* h, int Ls, const double* sigl, const double* x, double* y) {
    Oracle* o = static_cast<Oracle*>(h);
    if (o->sigt.empty() || o->sl.empty()) return 8;
    MomentSpace ms;
    moment_space_init(*o, ms, Ls);
    std::vector<double> scratch;
    Apply A = moment_operator(*o, ms, sigl, scratch);
    A(x, y);
    return 0;
}

// Within-group solve in moment space: b = D T^-1 (q + M s_mom) (q angular [NI][NENK] and s_mom
// moments [nm][NENK], either may be null), phi0 = b, GMRES(m) (pdiag null) or FGMRES(m) with the
// right preconditioner z_j = pdiag[j] v_j (iters.f:2511-2795), stopping test ||b - A phi|| <=
// rtol ||b|| + atol.  phi [nm][NENK] receives the solution; psi (optional) the angular flux
// T^-1 (M S phi + q + M s_mom).  Returns the gmres_sparskit status (0, -1 limit, -3 breakdown).
int or_moment_solve(void* h, int Ls, const double* sigl, const double* q, const double* s_mom, int m, double rtol,
                    double atol, int maxit, const double* pdiag, double* phi, double* psi, int* iters, double* resid,
                    double* history, int hist_len, int* hist_n) {
    Oracle* o = static_cast<Oracle*>(h);
    if (o->sigt.empty() || o->sl.empty()) return 8;
    MomentSpace ms;
    moment_space_init(*o, ms, Ls);
    const size_t n = (size_t)ms.nm * o->NENK;
    std::vector<double> b(n), scratch;
    moment_transport(*o, ms, s_mom, q, b.data(), nullptr);
    std::memcpy(phi, b.data(), sizeof(double) * n);
    Apply A = moment_operator(*o, ms, sigl, scratch);
    Apply P = [&ms, o, pdiag](const double* in, double* out) { moment_diag_precond(ms, o->NENK, pdiag, in, out); };
    std::vector<double> hist;
    int st = gmres_sparskit(n, b.data(), phi, m, rtol, atol, maxit, A, pdiag ? &P : nullptr, iters, resid, &hist);
    if (psi) {
        // psi = T^-1 (M (S phi + s_mom) + q)
        std::vector<double> sp(n);
        moment_scale(*o, ms, sigl, phi, sp.data());
        if (s_mom)
            for (size_t k2 = 0; k2 < n; ++k2) sp[k2] = sp[k2] + s_mom[k2];
        std::vector<double> y(n);
        moment_transport(*o, ms, sp.data(), q, y.data(), psi);
    }
    if (history && hist_n) {
        int c = std::min<int>(hist_len, (int)hist.size());
        for (int k2 = 0; k2 < c; ++k2) history[k2] = hist[k2];
        *hist_n = (int)hist.size();
    }
    return st;
}

// Multigroup dose solve in moment space: the group loop of Main.f90:326-476 with PIEISource
// (Main.f90:584-629) and the tally of CalculateDeposition (Main.f90:750-824, TallyDeposition.f90),
// on the same synthetic first-collision data as or_multigroup (uncollided flux u(r) of a
// monodirectional beam in group 0).  Per group g:
//   s_g = sum_{g'<g} S_{g'->g} phi_{g'} + S_{0->g} Y(Omega_b) u      (moment form of K psi_{g'} and of
//          the first-collision source sum_l s_l (2l+1)/(4 pi) P_l(k_i.Omega_b) u)
//   b_g = D T_g^-1 M s_g,  A_g phi_g = b_g by GMRES(m) from phi_g = b_g,
//   fluence_g = sqrt(4 pi) phi_g[0] (+ u for g = 0),  dose += dd[g][mat] fluence_g.
// sigt [G][Nm], sigs [G'][G][Nm][Ls+1] (transfer g' -> g), dd [G][Nm], unc [NENK], beam_dir [3].
// rtol_snap > rtol: each group is first solved to rtol_snap, its fluence stored in flux_snap (and
// dose_snap, iters_snap), then the same iterate is continued to rtol (flux, dose, iters); the
// groups below always see the rtol solution.  verbose prints one line per group to stderr.
int or_mg_moment(void* h, int G, int Ls, const double* sigt, const double* sigs, const double* dd, const double* unc,
                 const double* beam_dir, int m, double rtol, double rtol_snap, double atol, int maxit, double* flux,
                 double* dose, int* iters, double* flux_snap, double* dose_snap, int* iters_snap, int verbose) {
    Oracle* o = static_cast<Oracle*>(h);
    if (o->sl.empty()) return 8;
    const int Nm = o->Nm;
    const long NENK = o->NENK;
    MomentSpace ms;
    moment_space_init(*o, ms, Ls);
    const int nm = ms.nm;
    const size_t n = (size_t)nm * NENK;
    std::vector<std::vector<double>> phi_all(G);
    std::vector<double> src(n), b(n), scratch;
    std::vector<double> yb(nm);
    real_sh(Ls, beam_dir, yb.data());
    const double sq4pi = std::sqrt(FOURPI);
    for (long sd = 0; sd < NENK; ++sd) dose[sd] = 0.0;
    if (dose_snap) for (long sd = 0; sd < NENK; ++sd) dose_snap[sd] = 0.0;
    auto tsig = [&](int gp, int g) { return sigs + ((size_t)gp * G + g) * Nm * (Ls + 1); };
    for (int g = 0; g < G; ++g) {
        const double t0 = omp_get_wtime();
        // downscatter + first-collision source of group g
        const double* s0 = tsig(0, g);
#pragma omp parallel for schedule(static)
        for (long sd = 0; sd < NENK; ++sd) {
            const int mm = o->mat[sd / 4];
            for (int j = 0; j < nm; ++j) {
                double a = s0[(size_t)mm * (Ls + 1) + ms.lofj[j]] * yb[j] * unc[sd];
                for (int gp = 0; gp < g; ++gp)
                    a = a + tsig(gp, g)[(size_t)mm * (Ls + 1) + ms.lofj[j]] * phi_all[gp][(size_t)j * NENK + sd];
                src[(size_t)j * NENK + sd] = a;
            }
        }
        o->sigt.assign(sigt + (size_t)g * Nm, sigt + (size_t)(g + 1) * Nm);
        moment_transport(*o, ms, src.data(), nullptr, b.data(), nullptr);
        phi_all[g] = b;
        double* phi = phi_all[g].data();
        Apply A = moment_operator(*o, ms, tsig(g, g), scratch);
        int it = 0, it_snap = 0, st = 0;
        double res = 0.0;
        auto tally = [&](double* fl, double* ds) {
            for (long sd = 0; sd < NENK; ++sd) {
                double f = sq4pi * phi[sd];
                if (g == 0) f = f + unc[sd];
                fl[sd] = f;
                ds[sd] = ds[sd] + dd[(size_t)g * Nm + o->mat[sd / 4]] * f;
            }
        };
        if (rtol_snap > rtol && flux_snap && dose_snap) {
            st = gmres_sparskit(n, b.data(), phi, m, rtol_snap, atol, maxit, A, nullptr, &it_snap, &res, nullptr);
            if (st != 0) return 6;
            tally(flux_snap + (size_t)g * NENK, dose_snap);
            if (iters_snap) iters_snap[g] = it_snap;
        }
        st = gmres_sparskit(n, b.data(), phi, m, rtol, atol, maxit, A, nullptr, &it, &res, nullptr);
        if (st != 0) return 6;
        iters[g] = it + it_snap;
        tally(flux + (size_t)g * NENK, dose);
        if (verbose)
            std::fprintf(stderr, "group %2d: %3d + %3d operator applications, residual %.3e, %.1f s\n", g, it_snap, it,
                         res, omp_get_wtime() - t0);
    }
    return 0;
}


// ------------------------------------------------------------------------------------------
//  Planar beam, uncollided fluence at the DG nodes: RayTracing.f90:152-201 (quadrature points of
//  the elements in the field, ray from the point's projection Rp on the beam plane), TraceVector
//  RayTracing.f90:205-379 (Moller-Trumbore against every region-boundary face, per-material path
//  lengths from the sorted intersections; the single-material branch takes the one front-facing
//  boundary hit), InField.f90:47-63 (rectangle), FluenceQuadrature.f90:28-32 (Beer's law) and the
//  projection of FCSSource.f90:134-169 (phi0ek = M_ref^-1 sum_q w_q N_k(q) phi0q).  A region is the
//  set of elements of one material; its faces are the element faces on the mesh boundary or next to
//  another material.  The 4-point tetrahedral rule of the absent NittanyPhysics library
//  (PrepTetrahedralQuadrature) is restated from its published form: barycentric (a, b, b, b),
//  a = (5 + 3 sqrt 5)/20, b = (5 - sqrt 5)/20, weights 1/24 on the reference tetrahedron.
//  origin, axis, e1, e2 [3]: beam frame; w1, w2: field widths; attn [Nm]; unc [NENK] out.
// ------------------------------------------------------------------------------------------
int or_beam_uncollided(void* hp, const double* origin, const double* axis, const double* e1, const double* e2,
                       double w1, double w2, const double* attn, double* unc) {
    Oracle* o = static_cast<Oracle*>(hp);
    const int NE = o->NE, Nm = o->Nm;
    const double TOL = 1.0e-8, FTOL = 1.0e-12;
    const double qa = (5.0 + 3.0 * std::sqrt(5.0)) / 20.0, qb = (5.0 - std::sqrt(5.0)) / 20.0;
    // region faces: (element, local face) per material
    std::vector<std::vector<std::pair<int, int>>> rf(Nm);
    for (int e = 0; e < NE; ++e)
        for (int f = 0; f < 4; ++f) {
            const int n = o->nbr[(size_t)e * 4 + f];
            if (n < 0 || o->mat[n] != o->mat[e]) rf[o->mat[e]].push_back({e, f});
        }
    // reference-element mass matrix inverse (IMr) and shape functions at the points
    double Mi[16];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) Mi[i * 4 + j] = (i == j ? 2.0 : 1.0) / 120.0;
    invert(4, Mi);
    int status = 0;
#pragma omp parallel for schedule(dynamic, 64)
    for (int e = 0; e < NE; ++e) {
        double phiq[4], load[4] = {0, 0, 0, 0};
        for (int kq = 0; kq < 4; ++kq) {
            double v[3] = {0, 0, 0};
            for (int k = 0; k < 4; ++k)
                for (int d = 0; d < 3; ++d) v[d] += (k == kq ? qa : qb) * o->rg[(size_t)o->node[(size_t)e * 4 + k] * 3 + d];
            // InField, rectangle
            double u[3], vv[3];
            for (int d = 0; d < 3; ++d) u[d] = v[d] - origin[d];
            const double ua = dot3(u, axis);
            for (int d = 0; d < 3; ++d) vv[d] = u[d] - ua * axis[d];
            const bool in = std::fabs(dot3(vv, e1)) <= 0.5 * w1 + FTOL && std::fabs(dot3(vv, e2)) <= 0.5 * w2 + FTOL;
            phiq[kq] = 0.0;
            if (!in) continue;
            // Rp = origin + ((v - origin).e1) e1 + ((v - origin).e2) e2, r = v - Rp
            double Rp[3], r[3];
            const double a1 = dot3(u, e1), a2 = dot3(u, e2);
            for (int d = 0; d < 3; ++d) {
                Rp[d] = origin[d] + a1 * e1[d] + a2 * e2[d];
                r[d] = v[d] - Rp[d];
            }
            const double length = norm2_scaled(r, 3);
            std::vector<double> pathlen(Nm, 0.0);
            bool success = false;
            double tsingle = 0.0;
            for (int reg = 0; reg < Nm; ++reg) {
                std::vector<double> llist;
                for (auto [fe, ff] : rf[reg]) {
                    const double* v0 = &o->rg[(size_t)o->node[(size_t)fe * 4 + F2K[ff][0]] * 3];
                    const double* v1 = &o->rg[(size_t)o->node[(size_t)fe * 4 + F2K[ff][1]] * 3];
                    const double* v2 = &o->rg[(size_t)o->node[(size_t)fe * 4 + F2K[ff][2]] * 3];
                    double edge1[3], edge2[3], nref[3], pvec[3], tvec[3], qvec[3];
                    for (int d = 0; d < 3; ++d) { edge1[d] = v1[d] - v0[d]; edge2[d] = v2[d] - v0[d]; }
                    const double* n = &o->nrm[(size_t)fe * 12 + ff * 3];
                    double det = dot3(n, r);
                    if (Nm == 1) { if (det > -TOL) continue; }
                    else if (std::fabs(det) < TOL) continue;
                    cross3(edge1, edge2, nref);
                    if (dot3(n, nref) < 0.0)
                        for (int d = 0; d < 3; ++d) std::swap(edge1[d], edge2[d]);
                    cross3(r, edge2, pvec);
                    det = dot3(edge1, pvec);
                    if (std::fabs(det) < TOL) continue;
                    for (int d = 0; d < 3; ++d) tvec[d] = Rp[d] - v0[d];
                    const double uu = dot3(tvec, pvec);
                    cross3(tvec, edge1, qvec);
                    const double vq = dot3(r, qvec);
                    if (det > 0.0) {
                        if (uu < -TOL || uu > det + TOL) continue;
                        if (vq < -TOL || uu + vq > det + TOL) continue;
                    } else {
                        if (uu > TOL || uu < det - TOL) continue;
                        if (vq > TOL || uu + vq < det - TOL) continue;
                    }
                    const double t = dot3(edge2, qvec) / det;
                    if (Nm == 1) { success = true; tsingle = t; break; }
                    if (t > 1.0) continue;
                    llist.push_back(t);
                }
                if (Nm == 1) break;
                if (llist.size() == 1 && std::fabs(llist[0]) < 1.0e-12) continue;
                if (llist.empty()) continue;
                std::sort(llist.begin(), llist.end());
                size_t nkeep = 1;
                for (size_t i = 1; i < llist.size(); ++i)
                    if (std::fabs(llist[i] - llist[nkeep - 1]) > 1.0e-12) llist[nkeep++] = llist[i];
                llist.resize(nkeep);
                for (size_t il = 0; il + 1 < llist.size(); il += 2) pathlen[reg] += llist[il + 1] - llist[il];
                if (llist.size() % 2 == 1) pathlen[reg] += 1.0 - llist.back();
            }
            if (Nm == 1) {
                if (!success) {
#pragma omp critical
                    status = 1;
                    continue;
                }
                pathlen[0] = (1.0 - tsingle) * length;
            } else {
                for (int m = 0; m < Nm; ++m) pathlen[m] *= length;
            }
            double tau = 0.0;
            for (int m = 0; m < Nm; ++m) tau += attn[m] * pathlen[m];
            phiq[kq] = std::exp(-tau);
        }
        for (int k = 0; k < 4; ++k)
            for (int kq = 0; kq < 4; ++kq) load[k] += (1.0 / 24.0) * (k == kq ? qa : qb) * phiq[kq];
        for (int k = 0; k < 4; ++k) {
            double c = 0.0;
            for (int j = 0; j < 4; ++j) c += Mi[k * 4 + j] * load[j];
            unc[(size_t)e * 4 + k] = c;
        }
    }
    return status;
}

}  // extern "C"
