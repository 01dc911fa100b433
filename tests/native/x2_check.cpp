// Checks the two-lane fp32 forms of the packed 2D sweep (egg_b200/csrc/x2.cuh,
// compiled for the host with per-lane arithmetic) against the fp64 metric of
// metric.cuh:
//   roles2<KIND>     vs the role contraction of mu_eval<double> (both lanes,
//                    every role entry, signs of all four samples of a cell),
//   dmu2_pair<KIND>  vs dmu2<double> for moves of column 0, column 1 and of
//                    the corner (both columns).
// Prints "roles KIND err" and "dmu KIND err" lines: the worst error relative
// to the size of the quantity's terms.
#include <cmath>
#include <cstdio>
#include <random>

#include "x2.cuh"

using namespace egg_b200;

int main()
{
    std::mt19937_64 rng(11);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    for (int kind = 0; kind < 3; ++kind) {
        double w_roles = 0.0, w_dmu = 0.0;
        for (int it = 0; it < 4000; ++it) {
            const double h = std::pow(10.0, -3.0 * std::fabs(U(rng)));
            const double delta = kind == kUntangle ? 0.3 * h * h : 0.0;
            double T[2][4];
            for (int l = 0; l < 2; ++l) {
                const double t[4] = {h * (1.0 + 0.35 * U(rng)), h * 0.35 * U(rng), h * 0.35 * U(rng),
                                     h * (1.0 + 0.35 * U(rng))};
                for (int i = 0; i < 4; ++i) { T[l][i] = double(float(t[i])); }
            }
            const int pair = it & 1;  // samples (0,1) or (2,3): s0 = +-1, s1 = (1, -1)
            const double s0l[2] = {pair ? -1.0 : 1.0, pair ? -1.0 : 1.0}, s1l[2] = {1.0, -1.0};
            auto F2 = [&](int i) { return make_float2(float(T[0][i]), float(T[1][i])); };
            Roles2 o;
            const float fdelta = float(delta);
            switch (kind) {
            case kShape: roles2<kShape>(F2(0), F2(1), F2(2), F2(3), make_float2(float(s0l[0]), float(s0l[1])),
                                        make_float2(1.0f, -1.0f), fdelta, o); break;
            case kUntangle: roles2<kUntangle>(F2(0), F2(1), F2(2), F2(3), make_float2(float(s0l[0]), float(s0l[1])),
                                              make_float2(1.0f, -1.0f), fdelta, o); break;
            default: roles2<kShapeSize>(F2(0), F2(1), F2(2), F2(3), make_float2(float(s0l[0]), float(s0l[1])),
                                        make_float2(1.0f, -1.0f), fdelta, o); break;
            }
            for (int l = 0; l < 2; ++l) {
                double mu, g[4], H[16];
                mu_eval<double>(kind, T[l], delta, mu, g, H);
                const double s0 = s0l[l], s1 = s1l[l], ss = s0 * s1;
                const double r1[5] = {s0 * g[0], s0 * g[2], H[0], H[2], H[10]};
                const double r2[5] = {s1 * g[1], s1 * g[3], H[5], H[7], H[15]};
                const double r0[5] = {-(r1[0] + r2[0]), -(r1[1] + r2[1]), H[0] + H[5] + 2 * ss * H[1],
                                      H[2] + H[7] + ss * (H[3] + H[6]), H[10] + H[15] + 2 * ss * H[11]};
                double gs = 0.0, hs = 0.0;
                for (int i = 0; i < 4; ++i) { gs = std::fmax(gs, std::fabs(g[i])); }
                for (int i = 0; i < 16; ++i) { hs = std::fmax(hs, std::fabs(H[i])); }
                for (int q = 0; q < 5; ++q) {
                    const double sc = q < 2 ? gs : hs;
                    const float a0 = l ? o.r0[q].y : o.r0[q].x, a1 = l ? o.r1[q].y : o.r1[q].x;
                    const float a2 = l ? o.r2[q].y : o.r2[q].x;
                    w_roles = std::fmax(w_roles, std::fabs(a0 - r0[q]) / (2 * sc));
                    w_roles = std::fmax(w_roles, std::fabs(a1 - r1[q]) / sc);
                    w_roles = std::fmax(w_roles, std::fabs(a2 - r2[q]) / sc);
                }
            }
            // trial moves: column 0, column 1, corner
            const double dx = 0.05 * h * U(rng), dy = 0.05 * h * U(rng);
            for (int mv = 0; mv < 3; ++mv) {
                double dt[2][4];
                float2 ds, dD;
                float dsx[2], dDx[2];
                for (int l = 0; l < 2; ++l) {
                    const double e0x = mv == 1 ? 0.0 : (mv == 0 ? dx : -dx), e0y = mv == 1 ? 0.0 : (mv == 0 ? dy : -dy);
                    const double e1x = mv == 0 ? 0.0 : (mv == 1 ? dx : -dx), e1y = mv == 0 ? 0.0 : (mv == 1 ? dy : -dy);
                    dt[l][0] = e0x;
                    dt[l][1] = e1x;
                    dt[l][2] = e0y;
                    dt[l][3] = e1y;
                    const float* tf = nullptr;
                    (void)tf;
                    const float t0 = float(T[l][0]), t1 = float(T[l][1]), t2 = float(T[l][2]), t3 = float(T[l][3]);
                    const float fe0x = float(e0x), fe0y = float(e0y), fe1x = float(e1x), fe1y = float(e1y);
                    dsx[l] = 2.0f * ((t0 * fe0x + t2 * fe0y) + (t1 * fe1x + t3 * fe1y)) +
                             (fe0x * fe0x + fe0y * fe0y + fe1x * fe1x + fe1y * fe1y);
                    dDx[l] = (fe0x * t3 - fe0y * t1) + (t0 * fe1y - t2 * fe1x);
                }
                ds = make_float2(dsx[0], dsx[1]);
                dD = make_float2(dDx[0], dDx[1]);
                float2 s, D;
                {
                    float sv[2], Dv[2];
                    for (int l = 0; l < 2; ++l) {
                        const float t0 = float(T[l][0]), t1 = float(T[l][1]), t2 = float(T[l][2]), t3 = float(T[l][3]);
                        sv[l] = t0 * t0 + t1 * t1 + t2 * t2 + t3 * t3;
                        Dv[l] = t0 * t3 - t1 * t2;
                    }
                    s = make_float2(sv[0], sv[1]);
                    D = make_float2(Dv[0], Dv[1]);
                }
                const float2 twoD = add2(D, D);
                const float2 m2 = make_float2(s.x / D.x, s.y / D.y);
                float2 dn, dm;
                switch (kind) {
                case kShape: dm = dmu2_pair<kShape>(s, D, twoD, m2, ds, dD, fdelta, dn); break;
                case kUntangle: dm = dmu2_pair<kUntangle>(s, D, twoD, m2, ds, dD, fdelta, dn); break;
                default: dm = dmu2_pair<kShapeSize>(s, D, twoD, m2, ds, dD, fdelta, dn); break;
                }
                for (int l = 0; l < 2; ++l) {
                    double dnr;
                    const double ref = dmu2<double>(kind, T[l], dt[l], delta, dnr);
                    // scale: the first-order size of the change
                    double mu, g[4], H[16];
                    mu_eval<double>(kind, T[l], delta, mu, g, H);
                    double gn = 0.0;
                    for (int i = 0; i < 4; ++i) { gn += std::fabs(g[i] * dt[l][i]); }
                    const float got = l ? dm.y : dm.x;
                    w_dmu = std::fmax(w_dmu, std::fabs(got - ref) / std::fmax(gn, 1e-300));
                }
            }
        }
        std::printf("roles %d %.3e\n", kind, w_roles);
        std::printf("dmu %d %.3e\n", kind, w_dmu);
    }
    return 0;
}
