// Host construction of the order-4 diagonal-norm SBP operator tables that
// the kernels consume (see plane_march.cuh, AxisT).
//
// The stencils are the Mattsson-Nordstrom (2004) order-4 diagonal-norm
// operators that Diffinitive.jl's `standard_diagonal.toml` (order 4)
// provides to the reference (read at src/BP8.jl:195): norm weights
// 17/48, 59/48, 43/48, 49/48; D1 with 4-row closures; the compatible narrow
// D2; the third-order boundary derivative. Every row is formed in exact
// rational arithmetic (numerator/denominator pairs below) and rounded once.
#pragma once
#include <cmath>
#include <vector>

namespace eqd {

struct Rat { double num, den; double v() const { return num / den; } };

static const Rat kHw[4] = {{17, 48}, {59, 48}, {43, 48}, {49, 48}};
static const Rat kD1Int[5] = {{1, 12}, {-2, 3}, {0, 1}, {2, 3}, {-1, 12}};
static const Rat kD2Int[5] = {{-1, 12}, {4, 3}, {-5, 2}, {4, 3}, {-1, 12}};
static const Rat kD1Cl[4][6] = {
    {{-24, 17}, {59, 34}, {-4, 17}, {-3, 34}, {0, 1}, {0, 1}},
    {{-1, 2}, {0, 1}, {1, 2}, {0, 1}, {0, 1}, {0, 1}},
    {{4, 43}, {-59, 86}, {0, 1}, {59, 86}, {-4, 43}, {0, 1}},
    {{3, 98}, {0, 1}, {-59, 98}, {0, 1}, {32, 49}, {-4, 49}},
};
static const Rat kD2Cl[4][6] = {
    {{2, 1}, {-5, 1}, {4, 1}, {-1, 1}, {0, 1}, {0, 1}},
    {{1, 1}, {-2, 1}, {1, 1}, {0, 1}, {0, 1}, {0, 1}},
    {{-4, 43}, {59, 43}, {-110, 43}, {59, 43}, {-4, 43}, {0, 1}},
    {{-1, 49}, {0, 1}, {59, 49}, {-118, 49}, {64, 49}, {-4, 49}},
};
static const Rat kDb[4] = {{-11, 6}, {3, 1}, {-3, 2}, {1, 3}};

// Dense 1D operators of length n, spacing h (row-major n x n).
struct Dense1D {
    int n;
    double h;
    std::vector<double> D1, D2, W;   // W = D1 * D1
    double d1(int r, int c) const { return D1[(size_t)r * n + c]; }
    double d2(int r, int c) const { return D2[(size_t)r * n + c]; }
    double w(int r, int c) const { return W[(size_t)r * n + c]; }

    Dense1D(int n_, double h_) : n(n_), h(h_), D1((size_t)n_ * n_, 0.0), D2((size_t)n_ * n_, 0.0), W((size_t)n_ * n_, 0.0) {
        const double hi = 1.0 / h, hi2 = hi * hi;
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 6; ++c) {
                // Coefficient * (1/h) in one rounding each, as the reference's
                // operators scale each stencil entry by the inverse spacing.
                D1[(size_t)r * n + c] = kD1Cl[r][c].v() * hi;
                D1[(size_t)(n - 1 - r) * n + (n - 1 - c)] = -kD1Cl[r][c].v() * hi;
                D2[(size_t)r * n + c] = kD2Cl[r][c].v() * hi2;
                D2[(size_t)(n - 1 - r) * n + (n - 1 - c)] = kD2Cl[r][c].v() * hi2;
            }
        for (int r = 4; r < n - 4; ++r)
            for (int o = -2; o <= 2; ++o) {
                D1[(size_t)r * n + r + o] = kD1Int[o + 2].v() * hi;
                D2[(size_t)r * n + r + o] = kD2Int[o + 2].v() * hi2;
            }
        for (int r = 0; r < n; ++r)
            for (int m = std::max(0, r - 5); m <= std::min(n - 1, r + 5); ++m) {
                const double a = D1[(size_t)r * n + m];
                if (a == 0.0) continue;
                for (int c = std::max(0, m - 5); c <= std::min(n - 1, m + 5); ++c)
                    W[(size_t)r * n + c] += a * D1[(size_t)m * n + c];
            }
    }
};

template <typename T, typename AX>
void fill_axis(AX &a, int n, double h) {
    Dense1D M(n, h);
    const double hi = 1.0 / h, hi2 = hi * hi;
    for (int k = 0; k < 5; ++k) {
        a.d1_int[k] = (T)(kD1Int[k].v() * hi);
        a.d2_int[k] = (T)(kD2Int[k].v() * hi2);
    }
    // Interior W stencil: a row far from both ends (exists for n >= 17);
    // otherwise the convolution of the interior D1 stencil with itself.
    for (int o = -4; o <= 4; ++o) {
        double s = 0.0;
        for (int m = -2; m <= 2; ++m) {
            const int k = o - m;
            if (k >= -2 && k <= 2) s += (kD1Int[m + 2].v() * hi) * (kD1Int[k + 2].v() * hi);
        }
        a.w_int[o + 4] = (T)s;
    }
    auto d1i = [&](int r, int c) { int o = c - r; return (o >= -2 && o <= 2) ? kD1Int[o + 2].v() * hi : 0.0; };
    auto d2i = [&](int r, int c) { int o = c - r; return (o >= -2 && o <= 2) ? kD2Int[o + 2].v() * hi2 : 0.0; };
    auto wi = [&](int r, int c) { int o = c - r; return (o >= -4 && o <= 4) ? (double)a.w_int[o + 4] : 0.0; };
    auto in = [&](int c) { return c >= 0 && c < n; };
    for (int r = 0; r < 4; ++r)
        for (int k = 0; k < 6; ++k) {
            const int cL = k, rR = n - 1 - r, cR = n - 1 - k;
            a.d1_corrL[r][k] = (T)(in(cL) ? M.d1(r, cL) - d1i(r, cL) : 0.0);
            a.d2_corrL[r][k] = (T)(in(cL) ? M.d2(r, cL) - d2i(r, cL) : 0.0);
            a.d1_corrR[r][k] = (T)(in(cR) ? M.d1(rR, cR) - d1i(rR, cR) : 0.0);
            a.d2_corrR[r][k] = (T)(in(cR) ? M.d2(rR, cR) - d2i(rR, cR) : 0.0);
        }
    for (int r = 0; r < 6; ++r)
        for (int k = 0; k < 11; ++k) {
            const int cL = k, rR = n - 1 - r, cR = n - 1 - k;
            a.w_corrL[r][k] = (T)(in(cL) ? M.w(r, cL) - wi(r, cL) : 0.0);
            a.w_corrR[r][k] = (T)(in(cR) ? M.w(rR, cR) - wi(rR, cR) : 0.0);
        }
    for (int t = 0; t < 8; ++t) {
        const int r = t < 4 ? t : n - 1 - (t - 4);
        for (int o = -3; o <= 3; ++o) {
            const int c = r + o;
            a.d1_cl[t][o + 3] = (T)(in(c) ? M.d1(r, c) : 0.0);
            a.d2_cl[t][o + 3] = (T)(in(c) ? M.d2(r, c) : 0.0);
        }
    }
    for (int k = 0; k < 4; ++k) {
        a.dlo[k] = (T)(kDb[k].v() * hi);
        a.wq[k] = (T)kHw[k].v();
    }
}

}  // namespace eqd
