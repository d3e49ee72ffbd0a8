// DKI fits of the simulated signal: the shell-wise cumulant fit and the
// linear least-squares DKI fit that analysis/readRMS.m (:51-94) and
// analysis/readRMS_pgse.m (:60-101) apply to the output files, and the
// apparent diffusivity / kurtosis along directions from either fit
// (readRMS.m:105-117).  Host code: per timepoint a few small least-squares
// problems whose matrices do not depend on the timepoint, so each matrix is
// factored once (Householder QR) and applied to every timepoint's right-hand
// side.
//
// Every least-squares solve is MATLAB's A\y, including its basic solution for
// a rank-deficient A (where MATLAB also prints a warning): the shell fit of
// readRMS_pgse.m, whose intercept column makes each direction's system one
// rank short, depends on it.
#include <algorithm>
#include <array>
#include <cfloat>
#include <cmath>
#include <string>
#include <vector>

#include "rms_sim.h"

namespace rms {
namespace {

// readRMS.m:13-18: tensor multiplicities and index lists of the 6 second-order
// and 15 fourth-order elements
constexpr double kDcnt[6] = {1, 2, 2, 1, 2, 1};
constexpr double kWcnt[15] = {1, 4, 4, 6, 12, 6, 4, 12, 12, 4, 1, 4, 6, 4, 1};
constexpr int kDind[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
constexpr int kWind[15][4] = {{0, 0, 0, 0}, {0, 0, 0, 1}, {0, 0, 0, 2}, {0, 0, 1, 1}, {0, 0, 1, 2},
                              {0, 0, 2, 2}, {0, 1, 1, 1}, {0, 1, 1, 2}, {0, 1, 2, 2}, {0, 2, 2, 2},
                              {1, 1, 1, 1}, {1, 1, 1, 2}, {1, 1, 2, 2}, {1, 2, 2, 2}, {2, 2, 2, 2}};

void ndir2(const double* n, double* out) {   // readRMS.m:123-125
    for (int i = 0; i < 6; ++i) out[i] = n[kDind[i][0]] * n[kDind[i][1]];
}
void ndir4(const double* n, double* out) {   // readRMS.m:119-121
    for (int i = 0; i < 15; ++i) out[i] = n[kWind[i][0]] * n[kWind[i][1]] * n[kWind[i][2]] * n[kWind[i][3]];
}

// A \ y as MATLAB's backslash computes it for a rectangular A: Householder QR
// with column pivoting (Businger & Golub 1965; Golub & Van Loan, Matrix
// Computations, 4th ed., §5.4.2): at each step the remaining column of
// largest norm is taken; the rank r is the number of |r_kk| above
// max(m, n) eps |r_11|; the result is the basic solution, the triangular
// solve on the r pivoted columns, zeros elsewhere.  For a full-rank A (m >= n)
// that is the least-squares solution.  A is stored column-major; the
// reflectors overwrite its lower part.
class LeastSquares {
  public:
    void factor(int m, int n, std::vector<double> a) {
        m_ = m;
        n_ = n;
        a_ = std::move(a);
        const int kmax = std::min(m, n);
        tau_.assign(kmax, 0.0);
        rdiag_.assign(kmax, 0.0);
        perm_.resize(n);
        for (int j = 0; j < n; ++j) perm_[j] = j;
        nref_ = 0;
        for (int k = 0; k < kmax; ++k) {
            // pivot: the column whose rows k.. have the largest norm (first on ties)
            int p = k;
            double best = -1.0;
            for (int j = k; j < n; ++j) {
                double nj = 0.0;
                for (int i = k; i < m; ++i) nj = std::hypot(nj, a_[(size_t)j * m + i]);
                if (nj > best) {
                    best = nj;
                    p = j;
                }
            }
            if (best == 0.0) break;   // the rest is zero: rank k
            if (p != k) {
                std::swap_ranges(a_.begin() + (size_t)k * m, a_.begin() + (size_t)(k + 1) * m,
                                 a_.begin() + (size_t)p * m);
                std::swap(perm_[k], perm_[p]);
            }
            double* col = &a_[(size_t)k * m];
            const double alpha = col[k];
            const double beta = alpha > 0 ? -best : best;
            const double v0 = alpha - beta;
            for (int i = k + 1; i < m; ++i) col[i] /= v0;   // reflector v = (1, col[k+1..])
            tau_[k] = (beta - alpha) / beta;
            rdiag_[k] = beta;
            col[k] = beta;
            for (int j = k + 1; j < n; ++j) {
                double* cj = &a_[(size_t)j * m];
                double w = cj[k];
                for (int i = k + 1; i < m; ++i) w += col[i] * cj[i];
                w *= tau_[k];
                cj[k] -= w;
                for (int i = k + 1; i < m; ++i) cj[i] -= w * col[i];
            }
            nref_ = k + 1;
        }
        const double tol = nref_ ? std::max(m, n) * DBL_EPSILON * std::fabs(rdiag_[0]) : 0.0;
        rank_ = 0;
        while (rank_ < nref_ && std::fabs(rdiag_[rank_]) > tol) ++rank_;
    }

    int rank() const { return rank_; }

    // x[n] from y[m] (y is overwritten with Q^T y)
    void solve(double* y, double* x) const {
        for (int k = 0; k < nref_; ++k) {
            const double* col = &a_[(size_t)k * m_];
            double w = y[k];
            for (int i = k + 1; i < m_; ++i) w += col[i] * y[i];
            w *= tau_[k];
            y[k] -= w;
            for (int i = k + 1; i < m_; ++i) y[i] -= w * col[i];
        }
        for (int j = 0; j < n_; ++j) x[j] = 0.0;
        for (int k = rank_ - 1; k >= 0; --k) {
            double s = y[k];
            for (int j = k + 1; j < rank_; ++j) s -= a_[(size_t)j * m_ + k] * x[perm_[j]];
            x[perm_[k]] = s / rdiag_[k];
        }
    }

  private:
    int m_ = 0, n_ = 0, nref_ = 0, rank_ = 0;
    std::vector<double> a_, tau_, rdiag_;
    std::vector<int> perm_;
};

}  // namespace
}  // namespace rms

using namespace rms;

extern "C" {

int rms_dki_shell(int T, int m, const double* sig, const double* bvec, const double* bval, const double* td,
                  int intercept, double* dt) {
    if (T < 1 || m < 1 || !sig || !bvec || !bval || !td || !dt) return set_error(RMS_ERR_ARG, "bad argument");
    try {
        // unique(bvec, 'rows') and the rows of each (exact equality, as ismember)
        std::vector<std::array<double, 3>> dirs;
        std::vector<std::vector<int>> rows;
        for (int r = 0; r < m; ++r) {
            const std::array<double, 3> g{bvec[3 * r], bvec[3 * r + 1], bvec[3 * r + 2]};
            size_t j = 0;
            while (j < dirs.size() && dirs[j] != g) ++j;
            if (j == dirs.size()) {
                dirs.push_back(g);
                rows.emplace_back();
            }
            rows[j].push_back(r);
        }
        // numel(unique(bval))
        std::vector<double> bs(bval, bval + m);
        std::sort(bs.begin(), bs.end());
        const int nbval = (int)(std::unique(bs.begin(), bs.end()) - bs.begin());
        if (nbval < 2) return set_error(RMS_ERR_ARG, "the shell fit needs at least two distinct b-values");
        // per direction: [1] -b, b^2/6, ..., b^nbval/6 (readRMS.m:68, readRMS_pgse.m:76)
        const int off = intercept ? 1 : 0;
        const int ncol = nbval + off;
        const int nbvec = (int)dirs.size();
        std::vector<LeastSquares> shell(nbvec);
        std::vector<double> y, x(std::max(ncol, 1));
        for (int j = 0; j < nbvec; ++j) {
            const int mj = (int)rows[j].size();
            std::vector<double> a((size_t)mj * ncol);
            for (int i = 0; i < mj; ++i) {
                const double b = bval[rows[j][i]];
                if (intercept) a[i] = 1.0;
                a[(size_t)off * mj + i] = -b;
                for (int p = 2; p <= nbval; ++p) a[(size_t)(off + p - 1) * mj + i] = (1.0 / 6.0) * std::pow(b, p);
            }
            shell[j].factor(mj, ncol, std::move(a));
        }
        // n2 \ dx2g and n4 \ dx4g over the unique directions (readRMS.m:75-76)
        LeastSquares f2, f4;
        {
            std::vector<double> a2((size_t)nbvec * 6), a4((size_t)nbvec * 15);
            for (int j = 0; j < nbvec; ++j) {
                double n2[6], n4[15];
                ndir2(dirs[j].data(), n2);
                ndir4(dirs[j].data(), n4);
                for (int i = 0; i < 6; ++i) a2[(size_t)i * nbvec + j] = n2[i];
                for (int i = 0; i < 15; ++i) a4[(size_t)i * nbvec + j] = n4[i];
            }
            f2.factor(nbvec, 6, std::move(a2));
            f4.factor(nbvec, 15, std::move(a4));
        }
        std::vector<double> dx2g(nbvec), dx4g(nbvec), w(nbvec);
        for (int t = 0; t < T; ++t) {
            const double* st = sig + (size_t)t * m;
            for (int j = 0; j < nbvec; ++j) {
                y.resize(rows[j].size());
                for (size_t i = 0; i < rows[j].size(); ++i) y[i] = std::log(st[rows[j][i]] + DBL_EPSILON);
                shell[j].solve(y.data(), x.data());
                const double Dj = x[off], Kj = x[off + 1] / (x[off] * x[off]);
                dx2g[j] = Dj * 2.0 * td[t];
                dx4g[j] = (Kj + 3.0) * dx2g[j] * dx2g[j];
            }
            w = dx2g;
            f2.solve(w.data(), dt + (size_t)t * 21);
            w = dx4g;
            f4.solve(w.data(), dt + (size_t)t * 21 + 6);
        }
        return RMS_OK;
    } catch (const std::exception& e) {
        return set_error(RMS_ERR_NOMEM, e.what());
    }
}

int rms_dki_lls(int T, int m, const double* sig, const double* bvec, const double* bval, double* dt) {
    if (T < 1 || m < 1 || !sig || !bvec || !bval || !dt) return set_error(RMS_ERR_ARG, "bad argument");
    try {
        // readRMS.m:80-91: unit gradient directions (zero rows left zero),
        // -b g_i g_j D_cnt and b^2/6 g_i g_j g_k g_l W_cnt
        std::vector<double> a((size_t)m * 21);
        for (int r = 0; r < m; ++r) {
            double g[3] = {bvec[3 * r], bvec[3 * r + 1], bvec[3 * r + 2]};
            double norm = std::sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
            if (norm == 0.0) norm = 1.0;
            for (double& c : g) c /= norm;
            const double b = bval[r];
            double n2[6], n4[15];
            ndir2(g, n2);
            ndir4(g, n4);
            for (int i = 0; i < 6; ++i) a[(size_t)i * m + r] = -(b * n2[i]) * kDcnt[i];
            const double bsqd6 = b * b / 6.0;
            for (int i = 0; i < 15; ++i) a[(size_t)(6 + i) * m + r] = (bsqd6 * n4[i]) * kWcnt[i];
        }
        LeastSquares f;
        f.factor(m, 21, std::move(a));
        std::vector<double> y(m);
        for (int t = 0; t < T; ++t) {
            for (int r = 0; r < m; ++r) y[r] = std::log(sig[(size_t)t * m + r] + DBL_EPSILON);
            f.solve(y.data(), dt + (size_t)t * 21);
        }
        return RMS_OK;
    } catch (const std::exception& e) {
        return set_error(RMS_ERR_NOMEM, e.what());
    }
}

int rms_akc_shell(int T, const double* dt, int ndir, const double* dirs, const double* td, double* D, double* K) {
    if (T < 1 || ndir < 1 || !dt || !dirs || !td || !D || !K) return set_error(RMS_ERR_ARG, "bad argument");
    for (int q = 0; q < ndir; ++q) {
        double n2[6], n4[15];
        ndir2(dirs + 3 * q, n2);
        ndir4(dirs + 3 * q, n4);
        for (int t = 0; t < T; ++t) {
            // readRMS.m:105-112
            const double* row = dt + (size_t)t * 21;
            double x2 = 0.0, x4 = 0.0;
            for (int i = 0; i < 6; ++i) x2 += row[i] * n2[i];
            for (int i = 0; i < 15; ++i) x4 += row[6 + i] * n4[i];
            D[(size_t)t * ndir + q] = x2 / 2.0 / td[t];
            K[(size_t)t * ndir + q] = x4 / (x2 * x2) - 3.0;
        }
    }
    return RMS_OK;
}

int rms_akc_lls(int T, const double* dt, int ndir, const double* dirs, double* D, double* K) {
    if (T < 1 || ndir < 1 || !dt || !dirs || !D || !K) return set_error(RMS_ERR_ARG, "bad argument");
    for (int q = 0; q < ndir; ++q) {
        double n[3] = {dirs[3 * q], dirs[3 * q + 1], dirs[3 * q + 2]};
        const double norm = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        if (norm == 0.0) return set_error(RMS_ERR_ARG, "zero direction");
        for (double& c : n) c /= norm;
        double n2[6], n4[15];
        ndir2(n, n2);
        ndir4(n, n4);
        for (int t = 0; t < T; ++t) {
            // DKI signal model ln S = -b D(n) + b^2 D(n)^2 K(n) / 6 with the
            // coefficients of the fit above: D(n) = sum D_cnt c_i n_i n_j,
            // D(n)^2 K(n) = sum W_cnt c_ijkl n_i n_j n_k n_l
            const double* row = dt + (size_t)t * 21;
            double dn = 0.0, w = 0.0;
            for (int i = 0; i < 6; ++i) dn += kDcnt[i] * row[i] * n2[i];
            for (int i = 0; i < 15; ++i) w += kWcnt[i] * row[6 + i] * n4[i];
            D[(size_t)t * ndir + q] = dn;
            K[(size_t)t * ndir + q] = w / (dn * dn);
        }
    }
    return RMS_OK;
}

}  // extern "C"
