// Host FP64 generation of the NDG_t<LegendrePolynomial_t> tables.
//
// The device consumes these tables (constant memory per order); they are
// generated on the host in FP64 because they are a few KB, built once, and
// must match the reference bit for bit: the same algorithms (Kopriva,
// "Implementing Spectral Methods for PDEs", Algorithms 22, 23, 30, 34, 36,
// 37 and 57) evaluated in the same order as include/entities/NDG_t.tpp:10-59
// and src/polynomials/LegendrePolynomial_t.cpp. Compiled without FMA
// contraction so each product and sum rounds once, as in the reference.
#include "ndg_internal.hpp"

#include <cfloat>
#include <cmath>
#include <limits>

namespace ndg {
namespace {

constexpr double kPi = 3.14159265358979323846;

// Three-term recurrence for L_N and L_N' (Algorithm 22,
// src/polynomials/LegendrePolynomial_t.cpp:8-32).
struct LegendreValue {
    double value;
    double slope;
};

LegendreValue legendre(int N, double x) {
    if (N == 0) return {1.0, 0.0};
    if (N == 1) return {x, 1.0};
    double prev2 = 1.0, prev1 = x, prev2_slope = 0.0, prev1_slope = 1.0;
    LegendreValue out{0.0, 0.0};
    for (int k = 2; k <= N; ++k) {
        out.value = (2 * k - 1) * x * prev1 / k - (k - 1) * prev2 / k;
        out.slope = prev2_slope + (2 * k - 1) * prev1;
        prev2 = prev1;
        prev1 = out.value;
        prev2_slope = prev1_slope;
        prev1_slope = out.slope;
    }
    return out;
}

// Gauss-Legendre nodes and weights (Algorithm 23,
// src/polynomials/LegendrePolynomial_t.cpp:60-101): Newton iterations from
// the Chebyshev-Gauss guess, symmetric fill, exact middle node for even N.
void gauss_legendre(int N, std::vector<double>& x, std::vector<double>& w) {
    for (int i = 0; i < (N + 1) / 2; ++i) {
        if (N == 1) {
            x[0] = -std::sqrt(1.0 / 3.0);
            w[0] = 1.0;
            x[1] = -x[0];
            w[1] = w[0];
            continue;
        }
        double node = -std::cos(kPi * (2 * i + 1) / (2 * N + 2));
        for (int it = 0; it < 1000; ++it) {
            const LegendreValue L = legendre(N + 1, node);
            const double step = -L.value / L.slope;
            node += step;
            if (std::abs(step) <= std::numeric_limits<double>::min() * 2 * std::abs(node)) break;
        }
        const double slope = legendre(N + 1, node).slope;
        x[static_cast<size_t>(i)] = node;
        x[static_cast<size_t>(N - i)] = -node;
        w[static_cast<size_t>(i)] = 2.0 / ((1 - std::pow(node, 2)) * std::pow(slope, 2));
        w[static_cast<size_t>(N - i)] = w[static_cast<size_t>(i)];
    }
    if (N == 0) {
        x[0] = 0.0;
        w[0] = 2.0;
    }
    if (N % 2 == 0) {
        const double slope = legendre(N + 1, 0.0).slope;
        x[static_cast<size_t>(N / 2)] = 0.0;
        w[static_cast<size_t>(N / 2)] = 2 / std::pow(slope, 2);
    }
}

}  // namespace

// 2-ulp closeness test used by the reference for node coincidence
// (include/entities/NDG_t.tpp:200-208).
bool almost_equal(double x, double y) {
    return std::abs(x - y) <= std::numeric_limits<double>::epsilon() * std::abs(x + y) * 2 ||
           std::abs(x - y) < std::numeric_limits<double>::min();
}

Tables build_tables(int N_max, int64_t n_interp) {
    if (N_max < 0 || N_max > 64) fail(NDG_ERR_INVALID_ARG, "N_max must be in [0, 64]");
    if (n_interp < 2) fail(NDG_ERR_INVALID_ARG, "n_interpolation_points must be at least 2");
    Tables T;
    T.N_max = N_max;
    T.n_interp = n_interp;
    for (auto& v : T.t) v.resize(static_cast<size_t>(N_max + 1));

    for (int N = 0; N <= N_max; ++N) {
        const size_t n = static_cast<size_t>(N + 1);
        const size_t uN = static_cast<size_t>(N);
        auto& x = T.t[NDG_TABLE_NODES][uN];
        auto& w = T.t[NDG_TABLE_WEIGHTS][uN];
        auto& bw = T.t[NDG_TABLE_BARYCENTRIC_WEIGHTS][uN];
        auto& D = T.t[NDG_TABLE_DERIVATIVE_MATRICES][uN];
        auto& Dcg = T.t[NDG_TABLE_G_HAT_DERIVATIVE_MATRICES][uN];
        auto& Dhat = T.t[NDG_TABLE_DERIVATIVE_MATRICES_HAT][uN];
        auto& interp = T.t[NDG_TABLE_INTERPOLATION_MATRICES][uN];
        auto& poly = T.t[NDG_TABLE_POLYNOMIALS][uN];
        auto& lL = T.t[NDG_TABLE_LAGRANGE_LEFT][uN];
        auto& lR = T.t[NDG_TABLE_LAGRANGE_RIGHT][uN];
        auto& dL = T.t[NDG_TABLE_LAGRANGE_DERIVATIVE_LEFT][uN];
        auto& dR = T.t[NDG_TABLE_LAGRANGE_DERIVATIVE_RIGHT][uN];
        for (auto* v : {&x, &w, &bw, &lL, &lR, &dL, &dR}) v->assign(n, 0.0);
        for (auto* v : {&D, &Dcg, &Dhat, &poly}) v->assign(n * n, 0.0);
        interp.assign(n * static_cast<size_t>(n_interp), 0.0);

        gauss_legendre(N, x, w);

        // Barycentric weights, Algorithm 30 (NDG_t.tpp:176-188).
        for (size_t j = 0; j < n; ++j) {
            double prod = 1.0;
            for (size_t i = 0; i < n; ++i)
                if (i != j) prod *= x[j] - x[i];
            bw[j] = 1.0 / prod;
        }
        // Modal projection rows P_i(x_j) w_j (2i+1)/2 (NDG_t.tpp:328-334).
        for (size_t i = 0; i < n; ++i)
            for (size_t j = 0; j < n; ++j) {
                double P = 1.0;
                if (i == 1) P = x[j];
                if (i >= 2) {
                    double p2 = 1.0, p1 = x[j];
                    for (size_t k = 2; k <= i; ++k) {
                        P = (2 * static_cast<int>(k) - 1) * x[j] * p1 / static_cast<int>(k) - (static_cast<int>(k) - 1) * p2 / static_cast<int>(k);
                        p2 = p1;
                        p1 = P;
                    }
                }
                poly[i * n + j] = P * w[j] * (2 * static_cast<int>(i) + 1) * 0.5;
            }
        // Off-diagonal derivative matrix, Algorithm 37 (NDG_t.tpp:252-261).
        for (size_t i = 0; i < n; ++i)
            for (size_t j = 0; j < n; ++j)
                if (i != j) D[i * n + j] = bw[j] / (bw[i] * (x[i] - x[j]));
        // Equispaced output interpolation rows (NDG_t.tpp:301-325).
        for (int64_t r = 0; r < n_interp; ++r) {
            const double xr = 2.0 * r / (n_interp - 1) - 1.0;
            double* row = interp.data() + static_cast<size_t>(r) * n;
            bool exact = false;
            for (size_t k = 0; k < n; ++k) {
                row[k] = 0.0;
                if (almost_equal(xr, x[k])) {
                    row[k] = 1.0;
                    exact = true;
                }
            }
            if (!exact) {
                double total = 0.0;
                for (size_t k = 0; k < n; ++k) {
                    row[k] = bw[k] / (xr - x[k]);
                    total += row[k];
                }
                for (size_t k = 0; k < n; ++k) row[k] /= total;
            }
        }
        // Lagrange basis and its derivative at -1 and +1, Algorithms 34 and 36
        // (NDG_t.tpp:210-250), then their normalisations.
        const double ends[2] = {-1.0, 1.0};
        std::vector<double>* basis[2] = {&lL, &lR};
        std::vector<double>* slope[2] = {&dL, &dR};
        for (int s = 0; s < 2; ++s)
            for (size_t i = 0; i < n; ++i) (*basis[s])[i] = bw[i] / (ends[s] - x[i]);
        for (int s = 0; s < 2; ++s)
            for (size_t i = 0; i < n; ++i) (*slope[s])[i] = bw[i] / ((ends[s] - x[i]) * (ends[s] - x[i]));
        for (int s = 0; s < 2; ++s) {
            double sum = 0.0;
            for (size_t i = 0; i < n; ++i) sum += (*basis[s])[i];
            for (size_t i = 0; i < n; ++i) (*basis[s])[i] /= sum;
        }
        for (int s = 0; s < 2; ++s) {
            double sum = 0.0;
            for (size_t i = 0; i < n; ++i) sum += bw[i] / (ends[s] - x[i]);
            for (size_t i = 0; i < n; ++i) (*slope[s])[i] /= sum;
        }
        // Diagonal as the negative off-diagonal row sum (NDG_t.tpp:263-274).
        for (size_t i = 0; i < n; ++i) {
            double diag = 0.0;
            for (size_t j = 0; j < n; ++j)
                if (j != i) diag -= D[i * n + j];
            D[i * n + i] = diag;
        }
        // Continuous-Galerkin second-derivative matrix, Algorithm 57 (NDG_t.tpp:287-298).
        for (size_t j = 0; j < n; ++j)
            for (size_t m = 0; m < n; ++m) {
                double s = 0.0;
                for (size_t k = 0; k < n; ++k) s += D[k * n + m] * D[k * n + j] * w[k];
                Dcg[j * n + m] = s / w[j];
            }
        // Weak-form derivative D^_ij = -D_ji w_j / w_i (NDG_t.tpp:277-284).
        for (size_t i = 0; i < n; ++i)
            for (size_t j = 0; j < n; ++j) Dhat[i * n + j] = -D[j * n + i] * w[j] / w[i];
    }
    return T;
}

}  // namespace ndg
