// Checks the forms that leave out known-zero terms (egg_b200/csrc/metric*.cuh,
// compiled for the host) against the general forms they replace:
//   dmu2_col<COL>            vs dmu2 with the zero entries of dT passed in,
//   role3(..., ax)           vs role3 with v = v[ax] e_ax passed in full,
//   line_sample3(..., ax)    vs line_sample3 with the full v,
//   line_norms3(..., ax)     vs line_norms3 with the full coefficients.
// Prints one line per check: its name and the worst relative difference.
#include <cmath>
#include <cstdio>
#include <random>

#include "metric3.cuh"

using namespace egg_b200;

static double rel(double a, double b) { return std::fabs(a - b) / std::fmax(1e-300, std::fmax(std::fabs(a), std::fabs(b))); }

int main()
{
    std::mt19937_64 rng(7);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    double w_col = 0, w_role = 0, w_line = 0, w_norm = 0;
    for (int kind = 0; kind < 3; ++kind) {
        for (int it = 0; it < 2000; ++it) {
            // 2D: a well-shaped T plus noise; a column move
            double t[4] = {1.0 + 0.3 * U(rng), 0.3 * U(rng), 0.3 * U(rng), 1.0 + 0.3 * U(rng)};
            const double ex = 0.05 * U(rng), ey = 0.05 * U(rng);
            for (int col = 0; col < 2; ++col) {
                double dt[4] = {0, 0, 0, 0};
                dt[col] = ex;
                dt[2 + col] = ey;
                double dn0, dn1;
                const double g = dmu2<double>(kind, t, dt, 0.01, dn0);
                const double c = col == 0 ? dmu2_col<double, 0>(kind, t, ex, ey, 0.01, dn1)
                                          : dmu2_col<double, 1>(kind, t, ex, ey, 0.01, dn1);
                w_col = std::fmax(w_col, std::fmax(rel(g, c), rel(dn0, dn1)));
            }
            // 3D
            double t3[9];
            for (int k = 0; k < 9; ++k) { t3[k] = (k % 4 == 0 ? 1.0 : 0.0) + 0.3 * U(rng); }
            Shared3<double> S;
            shared3<double>(kind, t3, 0.01, S);
            const double u[3] = {0.05 * U(rng), 0.05 * U(rng), 0.05 * U(rng)};
            for (int ax = 0; ax < 3; ++ax) {
                double v[3] = {0, 0, 0};
                v[ax] = U(rng) < 0 ? -1.0 : 1.0;
                double g0[3], h0[6], g1[3], h1[6];
                role3<double>(kind, S, v, g0, h0);
                role3<double>(kind, S, v, g1, h1, ax);
                for (int q = 0; q < 3; ++q) { w_role = std::fmax(w_role, rel(g0[q], g1[q])); }
                for (int q = 0; q < 6; ++q) { w_role = std::fmax(w_role, rel(h0[q], h1[q])); }
                LineSample3<double> L0, L1;
                line_sample3<double>(t3, u, v, L0);
                line_sample3<double>(t3, u, v, L1, ax);
                const double a0[8] = {L0.D, L0.D1, L0.s, L0.s1, L0.s2, L0.q, L0.q1, L0.q2};
                const double a1[8] = {L1.D, L1.D1, L1.s, L1.s1, L1.s2, L1.q, L1.q1, L1.q2};
                for (int q = 0; q < 8; ++q) { w_line = std::fmax(w_line, rel(a0[q], a1[q])); }
                for (double al : {1.0, 0.5, 0.125}) {
                    double n0[3], n1[3];
                    line_norms3<double>(L0, al, n0);
                    line_norms3<double>(L1, al, n1, ax);
                    for (int k = 0; k < 3; ++k) { w_norm = std::fmax(w_norm, rel(n0[k], n1[k])); }
                }
            }
        }
    }
    std::printf("dmu2_col %.3e\nrole3_ax %.3e\nline_sample3_ax %.3e\nline_norms3_ax %.3e\n", w_col, w_role, w_line,
                w_norm);
    return 0;
}
