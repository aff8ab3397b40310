// Host-side bookkeeping of restarted GMRES / FGMRES: Hessenberg columns, Givens rotations and the
// back-substitution, following SPARSKIT gmres/fgmres (third_party/SPARSKIT/iters.f:1901-2206,
// 2511-2795; givens :3225-3262).  The device does the vector work; one instance per problem.
#pragma once
#include <cmath>
#include <vector>

namespace lb {

// Givens rotation of SPARSKIT givens (iters.f:3225-3262): c, s with (x, y) -> (r, 0); on return
// x = r = |x_in * y'|.  When neither |y| > |x| nor |y| <= |x| holds (x or y is NaN) the rotation is
// the identity and r = 0, as in the reference.
inline void givens_rotation(double& x, double& y, double& c, double& s) {
    if (x == 0.0 && y == 0.0) {
        c = 1.0;
        s = 0.0;
    } else if (std::fabs(y) > std::fabs(x)) {
        const double t = x / y;
        x = std::sqrt(1.0 + t * t);
        s = std::copysign(1.0 / x, y);
        c = t * s;
    } else if (std::fabs(y) <= std::fabs(x)) {
        const double t = y / x;
        y = std::sqrt(1.0 + t * t);
        c = std::copysign(1.0 / y, x);
        s = t * c;
    } else {
        x = 0.0;
        y = 0.0;
        c = 1.0;
        s = 0.0;
    }
    x = std::fabs(x * y);
}

struct GmresHost {
    int m = 0;
    std::vector<std::vector<double>> H;   // H[col][row], 1-based rows as in SPARSKIT
    std::vector<double> c, s, rs;

    explicit GmresHost(int m_ = 0) { resize(m_); }

    void resize(int m_) {
        m = m_;
        H.assign(m + 2, std::vector<double>(m + 2, 0.0));
        c.assign(m + 2, 0.0);
        s.assign(m + 2, 0.0);
        rs.assign(m + 2, 0.0);
    }

    // start of a cycle with residual norm alpha
    void start(double alpha) { rs[1] = alpha; }

    // Column k (1-based) with projections hh[0..k-1] on v_1..v_k and subdiagonal hk: applies the
    // previous rotations, forms the new one (SPARSKIT givens) and returns |rs[k+1]|, the residual
    // estimate after k steps.
    double add_column(int k, const double* hh, double hk) {
        for (int i = 0; i < k; ++i) H[k][i + 1] = hh[i];
        H[k][k + 1] = hk;
        for (int i = 1; i <= k - 1; ++i) {
            const double a = H[k][i];
            H[k][i] = c[i] * a + s[i] * H[k][i + 1];
            H[k][i + 1] = c[i] * H[k][i + 1] - s[i] * a;
        }
        double x = H[k][k], y = H[k][k + 1], cc, ss;
        givens_rotation(x, y, cc, ss);
        H[k][k] = x;
        H[k][k + 1] = 0.0;
        c[k] = cc;
        s[k] = ss;
        const double a = -ss * rs[k];
        rs[k] = cc * rs[k];
        rs[k + 1] = a;
        return std::fabs(a);
    }

    // Back-substitution over the first k columns, dropping trailing columns with a zero diagonal.
    // Returns the number of columns kept (0: nothing to update) and the solution-update
    // coefficients coef[i] = -y_i (for the multi-axpy x -= sum coef_i v_i).
    int solve(int k, std::vector<double>& coef) {
        while (k > 0 && H[k][k] == 0.0) --k;
        coef.clear();
        if (k == 0) return 0;
        rs[k] = rs[k] / H[k][k];
        for (int i = k - 1; i >= 1; --i) {
            for (int ii = 1; ii <= i; ++ii) rs[ii] = rs[ii] - rs[i + 1] * H[i + 1][ii];
            rs[i] = rs[i] / H[i][i];
        }
        coef.resize(k);
        for (int i = 0; i < k; ++i) coef[i] = -rs[i + 1];
        return k;
    }
};

// Solves G c = hh for the k x k Gram matrix G of the Arnoldi basis (row stride ld) by Cholesky; G is
// the identity up to the basis' loss of orthogonality.  Returns false (c untouched) if G is not
// numerically positive definite.
inline bool gram_solve(const std::vector<double>& G, int ld, int k, const double* hh, double* c) {
    std::vector<double> L((size_t)k * k, 0.0);
    for (int j = 0; j < k; ++j) {
        double d = G[(size_t)j * ld + j];
        for (int p = 0; p < j; ++p) d -= L[(size_t)j * k + p] * L[(size_t)j * k + p];
        if (!(d > 0.5)) return false;   // G = I + E with |E| << 1 for any usable basis
        const double ljj = std::sqrt(d);
        L[(size_t)j * k + j] = ljj;
        for (int i = j + 1; i < k; ++i) {
            double t = G[(size_t)i * ld + j];
            for (int p = 0; p < j; ++p) t -= L[(size_t)i * k + p] * L[(size_t)j * k + p];
            L[(size_t)i * k + j] = t / ljj;
        }
    }
    std::vector<double> y(k);
    for (int i = 0; i < k; ++i) {
        double t = hh[i];
        for (int p = 0; p < i; ++p) t -= L[(size_t)i * k + p] * y[p];
        y[i] = t / L[(size_t)i * k + i];
    }
    for (int i = k - 1; i >= 0; --i) {
        double t = y[i];
        for (int p = i + 1; p < k; ++p) t -= L[(size_t)p * k + i] * c[p];
        c[i] = t / L[(size_t)i * k + i];
    }
    return true;
}

}  // namespace lb
