// Checks the difference forms dmu2 / dmu3 (egg_b200/csrc/metric*.cuh, compiled
// for the host) against differences of the metric evaluated in long double,
// and shows what they buy in fp32: prints, per objective and dimension, the
// worst relative error of the fp64 difference form, of the fp32 difference
// form, and of the naive fp32 difference mu(T + dT) - mu(T).
#include <cmath>
#include <cstdio>
#include <random>

#include "metric3.cuh"

using namespace egg_b200;

template <class L> static L mu2l(int kind, const L* a, double delta)
{
    const L D = a[0] * a[3] - a[1] * a[2], s = a[0] * a[0] + a[1] * a[1] + a[2] * a[2] + a[3] * a[3];
    if (kind == kShape) { return s / (2 * D) - 1; }
    if (kind == kUntangle) { return s / (2 * (0.5L * (D + sqrtl(D * D + 4.0L * delta * delta)))) - 1; }
    const L m = s / (2 * D);
    return m * m - 1 + (D - 1) * (D - 1);
}

template <class L> static L mu3l(int kind, const L* a, double delta)
{
    L C[9] = {a[4] * a[8] - a[5] * a[7], a[5] * a[6] - a[3] * a[8], a[3] * a[7] - a[4] * a[6],
              a[2] * a[7] - a[1] * a[8], a[0] * a[8] - a[2] * a[6], a[1] * a[6] - a[0] * a[7],
              a[1] * a[5] - a[2] * a[4], a[2] * a[3] - a[0] * a[5], a[0] * a[4] - a[1] * a[3]};
    L s = 0, q = 0;
    for (int k = 0; k < 9; ++k) {
        s += a[k] * a[k];
        q += C[k] * C[k];
    }
    const L D = a[0] * C[0] + a[1] * C[1] + a[2] * C[2];
    const L x = kind == kUntangle ? 0.5L * (D + sqrtl(D * D + 4.0L * delta * delta)) : D;
    L mu = s * q / (9 * x * x) - 1;
    if (kind == kShapeSize) { mu += (D - 1) * (D - 1); }
    return mu;
}

int main()
{
    std::mt19937_64 rng(11);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    for (int kind = 0; kind < 3; ++kind) {
        double e64[2] = {0, 0}, e32[2] = {0, 0}, naive[2] = {0, 0};
        for (int it = 0; it < 6000; ++it) {
            const double h = it % 2 ? 1e-3 : 1.0;  // unit cells and small cells
            // 2D
            double t[4] = {h * (1 + 0.3 * U(rng)), h * 0.3 * U(rng), h * 0.3 * U(rng), h * (1 + 0.3 * U(rng))};
            double dt[4];
            for (double& v : dt) { v = h * 1e-3 * U(rng); }
            const double delta2 = kind == kUntangle ? 0.1 * h * h : 0.0;
            float tf[4], dtf[4], tn[4];
            long double a[4], b[4], af[4], bf[4];
            for (int k = 0; k < 4; ++k) {
                tf[k] = float(t[k]);
                dtf[k] = float(dt[k]);
                tn[k] = tf[k] + dtf[k];
                a[k] = t[k];
                b[k] = (long double)t[k] + dt[k];
                af[k] = tf[k];
                bf[k] = (long double)tf[k] + dtf[k];
            }
            long double ref = mu2l(kind, b, delta2) - mu2l(kind, a, delta2);
            long double reff = mu2l(kind, bf, delta2) - mu2l(kind, af, delta2);
            double dn;
            float dnf;
            const double d64 = dmu2<double>(kind, t, dt, delta2, dn);
            const float d32 = dmu2<float>(kind, tf, dtf, float(delta2), dnf);
            const float nv = mu_value<float>(kind, tn, float(delta2)) - mu_value<float>(kind, tf, float(delta2));
            e64[0] = std::fmax(e64[0], std::fabs(double((d64 - ref) / ref)));
            e32[0] = std::fmax(e32[0], std::fabs(double((d32 - reff) / reff)));
            naive[0] = std::fmax(naive[0], std::fabs(double((nv - reff) / reff)));
            // 3D
            double t3[9], dt3[9];
            float t3f[9], dt3f[9], tn3[9];
            long double a3[9], b3[9], a3f[9], b3f[9];
            for (int k = 0; k < 9; ++k) {
                t3[k] = h * ((k % 4 == 0 ? 1.0 : 0.0) + 0.25 * U(rng));
                dt3[k] = h * 1e-3 * U(rng);
                t3f[k] = float(t3[k]);
                dt3f[k] = float(dt3[k]);
                tn3[k] = t3f[k] + dt3f[k];
                a3[k] = t3[k];
                b3[k] = (long double)t3[k] + dt3[k];
                a3f[k] = t3f[k];
                b3f[k] = (long double)t3f[k] + dt3f[k];
            }
            const double delta3 = kind == kUntangle ? 0.1 * h * h * h : 0.0;
            ref = mu3l(kind, b3, delta3) - mu3l(kind, a3, delta3);
            reff = mu3l(kind, b3f, delta3) - mu3l(kind, a3f, delta3);
            const double e3 = dmu3<double>(kind, t3, dt3, delta3, dn);
            const float f3 = dmu3<float>(kind, t3f, dt3f, float(delta3), dnf);
            float dd;
            const float nv3 = mu3_value<float>(kind, tn3, float(delta3), dd) - mu3_value<float>(kind, t3f, float(delta3), dd);
            e64[1] = std::fmax(e64[1], std::fabs(double((e3 - ref) / ref)));
            e32[1] = std::fmax(e32[1], std::fabs(double((f3 - reff) / reff)));
            naive[1] = std::fmax(naive[1], std::fabs(double((nv3 - reff) / reff)));
        }
        for (int d = 0; d < 2; ++d) {
            std::printf("%d %d %.3e %.3e %.3e\n", kind, d + 2, e64[d], e32[d], naive[d]);
        }
    }
    return 0;
}
