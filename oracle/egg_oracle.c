/* CPU oracle for the egg structured TMOP sweep -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's 2D block-Jacobi Newton vertex sweep
 * over explicit per-DOF patches (the "unstructured" form of the sweep: every
 * node has one position, so the frozen-halo structured store of the reference
 * and this global array see the same snapshot each sweep).  Used by the tests
 * and by bench.py's cpu_baseline leg as the parity checker; never by the
 * product.  Parity is pinned in tests/ against the reference's golden vectors
 * (tests/golden/) and against the reference core built from source
 * (oracle/_ref, see oracle/build_ref.sh).
 *
 * Reference algorithm followed:
 *   metric values / closed-form derivatives   src/metric.hpp:38-197
 *     (untangle: the reference differentiates by dual numbers,
 *      src/metric.hpp:924-982; here a closed form of the same function)
 *   A -> T -> det A per sample                  src/patch.hpp:95-117
 *   role-selected gradient / Hessian contraction src/patch.hpp:204-320
 *   patch evaluation order                      src/patch.hpp:325-346
 *   2x2 Newton solve with fallbacks             src/solve.hpp:32-46
 *   backtracking + acceptance + omega blend     src/sweep.hpp:1583-1648
 *   energy / min-det reduction                  src/sweep.hpp:1881-1922
 *   report cadence, double buffering            src/sweep.hpp:2027-2099
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

enum { K_SHAPE = 0, K_UNTANGLE = 1, K_SHAPE_SIZE = 2 };

typedef struct {
    double f, fp, fpp;
} scale_t;

static double det4(const double t[4]) { return t[0] * t[3] - t[1] * t[2]; }

static double mu_value(int kind, const double t[4], double delta)
{
    const double D = det4(t);
    const double s = t[0] * t[0] + t[1] * t[1] + t[2] * t[2] + t[3] * t[3];
    if (kind == K_SHAPE) return s / (2.0 * D) - 1.0;
    if (kind == K_UNTANGLE) {
        const double Dh = 0.5 * (D + sqrt(D * D + 4.0 * delta * delta));
        return s / (2.0 * Dh) - 1.0;
    }
    {
        const double m = s / (2.0 * D);
        return m * m - 1.0 + (D - 1.0) * (D - 1.0);
    }
}

/* mu = s f(D) (+ size term): gradient 2 f t + s f' cof, Hessian
 * 2 f I + 2 f'(t cof^T + cof t^T) + s f'' cof cof^T + s f' P. */
static void mu_eval(int kind, const double t[4], double delta, double* mu, double g[4], double H[16])
{
    static const double P[16] = {0, 0, 0, 1, 0, 0, -1, 0, 0, -1, 0, 0, 1, 0, 0, 0};
    const double D = det4(t);
    const double s = t[0] * t[0] + t[1] * t[1] + t[2] * t[2] + t[3] * t[3];
    const double cof[4] = {t[3], -t[2], -t[1], t[0]};
    scale_t sf;
    if (kind == K_UNTANGLE) {
        const double r = sqrt(D * D + 4.0 * delta * delta);
        const double Dh = 0.5 * (D + r);
        const double d1 = Dh / r, d2 = 2.0 * delta * delta / (r * r * r);
        sf.f = 0.5 / Dh;
        sf.fp = -0.5 * d1 / (Dh * Dh);
        sf.fpp = -0.5 * d2 / (Dh * Dh) + d1 * d1 / (Dh * Dh * Dh);
    } else {
        sf.f = 0.5 / D;
        sf.fp = -0.5 / (D * D);
        sf.fpp = 1.0 / (D * D * D);
    }
    const double m = s * sf.f;
    double g2[4], H2[16];
    for (int i = 0; i < 4; ++i) g2[i] = 2.0 * sf.f * t[i] + s * sf.fp * cof[i];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j)
            H2[i * 4 + j] = (i == j ? 2.0 * sf.f : 0.0) + 2.0 * sf.fp * (t[i] * cof[j] + cof[i] * t[j]) +
                            s * sf.fpp * cof[i] * cof[j] + s * sf.fp * P[i * 4 + j];
    if (kind != K_SHAPE_SIZE) {
        *mu = m - 1.0;
        memcpy(g, g2, sizeof g2);
        memcpy(H, H2, sizeof H2);
        return;
    }
    const double dm1 = D - 1.0;
    *mu = m * m - 1.0 + dm1 * dm1;
    for (int i = 0; i < 4; ++i) g[i] = 2.0 * m * g2[i] + 2.0 * dm1 * cof[i];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j)
            H[i * 4 + j] = 2.0 * g2[i] * g2[j] + 2.0 * m * H2[i * 4 + j] + 2.0 * cof[i] * cof[j] + 2.0 * dm1 * P[i * 4 + j];
}

/* A[:,k] = s_k (nbr_k - corner), T = A W (row-major), det A. */
static void sample_T(const double* c, const double* n0, const double* n1, double s0, double s1, const double* w,
                     double t[4], double* detA)
{
    double A[4];
    A[0] = s0 * (n0[0] - c[0]);
    A[1] = s1 * (n1[0] - c[0]);
    A[2] = s0 * (n0[1] - c[1]);
    A[3] = s1 * (n1[1] - c[1]);
    *detA = A[0] * A[3] - A[1] * A[2];
    for (int i = 0; i < 2; ++i)
        for (int k = 0; k < 2; ++k) {
            double acc = 0.0;
            for (int j = 0; j < 2; ++j) acc += A[i * 2 + j] * w[j * 2 + k];
            t[2 * i + k] = acc;
        }
}

typedef struct {
    int64_t ndof;
    const int32_t* dof;  /* [ndof] node id */
    const int64_t* off;  /* [ndof+1] */
    const int32_t* gc;   /* [occ] */
    const int32_t* gn0;
    const int32_t* gn1;
    const double* s0;
    const double* s1;
    const int32_t* role;
    const double* W;     /* [occ*4] */
    const double* wt;    /* [occ] or NULL (unit) */
} patches_t;

static void patch_eval(const patches_t* P, int64_t d, const double* X, int kind, double delta, double g[2],
                       double h[4], double* e, double* md)
{
    g[0] = g[1] = 0.0;
    h[0] = h[1] = h[2] = h[3] = 0.0;
    *e = 0.0;
    *md = INFINITY;
    for (int64_t p = P->off[d]; p < P->off[d + 1]; ++p) {
        const double* w = P->W + 4 * p;
        const double s0 = P->s0[p], s1 = P->s1[p];
        const double sv[2] = {s0, s1};
        double t[4], detA, mu, gg[4], H[16];
        sample_T(X + 2 * (int64_t)P->gc[p], X + 2 * (int64_t)P->gn0[p], X + 2 * (int64_t)P->gn1[p], s0, s1, w, t, &detA);
        if (detA < *md) *md = detA;
        const double wt = P->wt ? P->wt[p] : 1.0;
        mu_eval(kind, t, delta, &mu, gg, H);
        *e += wt * mu;
        const int role = P->role[p];
        /* gradient: dmu/dA[i,k] = sum_j g[i,j] w[k,j]; corner -sum_k s_k dA[i,k]; nbr s_ax dA[i,ax] */
        double dA[2][2];
        for (int i = 0; i < 2; ++i)
            for (int k = 0; k < 2; ++k) dA[i][k] = gg[i * 2 + 0] * w[k * 2 + 0] + gg[i * 2 + 1] * w[k * 2 + 1];
        double c[2] = {0.0, 0.0};
        if (role == 0) {
            for (int i = 0; i < 2; ++i) c[i] = -(sv[0] * dA[i][0] + sv[1] * dA[i][1]);
        } else if (role >= 1) {
            for (int i = 0; i < 2; ++i) c[i] = sv[role - 1] * dA[i][role - 1];
        }
        g[0] += wt * c[0];
        g[1] += wt * c[1];
        if (role < 0) continue;
        /* Jb (4x2): row a = (i, cc) has its only nonzero in column i. */
        double Jb[8] = {0};
        for (int a = 0; a < 4; ++a) {
            const int i = a / 2, cc = a % 2;
            double v;
            if (role == 0)
                v = -(sv[0] * w[0 * 2 + cc] + sv[1] * w[1 * 2 + cc]);
            else
                v = sv[role - 1] * w[(role - 1) * 2 + cc];
            Jb[a * 2 + i] = v;
        }
        for (int i = 0; i < 2; ++i)
            for (int j = 0; j < 2; ++j) {
                double acc = 0.0;
                for (int a = 0; a < 4; ++a) {
                    double hb = 0.0;
                    for (int b = 0; b < 4; ++b) hb += H[a * 4 + b] * Jb[b * 2 + j];
                    acc += Jb[a * 2 + i] * hb;
                }
                h[i * 2 + j] += wt * acc;
            }
    }
}

static void trial_eval(const patches_t* P, int64_t d, const double* X, int node, const double tr[2], int kind,
                       double delta, double* e, double* md)
{
    *e = 0.0;
    *md = INFINITY;
    for (int64_t p = P->off[d]; p < P->off[d + 1]; ++p) {
        const int ic = P->gc[p], i0 = P->gn0[p], i1 = P->gn1[p];
        const double* c = ic == node ? tr : X + 2 * (int64_t)ic;
        const double* n0 = i0 == node ? tr : X + 2 * (int64_t)i0;
        const double* n1 = i1 == node ? tr : X + 2 * (int64_t)i1;
        double t[4], detA;
        sample_T(c, n0, n1, P->s0[p], P->s1[p], P->W + 4 * p, t, &detA);
        *e += (P->wt ? P->wt[p] : 1.0) * mu_value(kind, t, delta);
        if (detA < *md) *md = detA;
    }
}

static void solve2(const double H[4], const double g[2], double x[2])
{
    const double gn = sqrt(g[0] * g[0] + g[1] * g[1]);
    if (gn < 1e-15) {
        x[0] = x[1] = 0.0;
        return;
    }
    const double inv = 1.0 / (H[0] * H[3] - H[1] * H[2]);
    x[0] = -inv * (H[3] * g[0] - H[1] * g[1]);
    x[1] = -inv * (-H[2] * g[0] + H[0] * g[1]);
    if (!(isfinite(x[0]) && isfinite(x[1]))) {
        const double c = -0.1 / gn;
        x[0] = c * g[0];
        x[1] = c * g[1];
    }
}

/* One DOF update from snapshot X into Xo. */
static void update_dof(const patches_t* P, int64_t d, const double* X, double* Xo, int kind, double delta, double omega)
{
    const int node = P->dof[d];
    const double pos[2] = {X[2 * node], X[2 * node + 1]};
    double g[2], h[4], e0, md0, dl[2];
    patch_eval(P, d, X, kind, delta, g, h, &e0, &md0);
    solve2(h, g, dl);
    double alpha = 1.0, cur[2] = {pos[0], pos[1]};
    for (int it = 0; it < 10; ++it) {
        const double tr[2] = {pos[0] + alpha * dl[0], pos[1] + alpha * dl[1]};
        double e, md;
        trial_eval(P, d, X, node, tr, kind, delta, &e, &md);
        const int ok = isfinite(e) && e <= e0 + 1e-12 && (kind == K_UNTANGLE || md > 0.0);
        if (ok) {
            cur[0] = tr[0];
            cur[1] = tr[1];
            break;
        }
        alpha *= 0.5;
    }
    if (omega != 1.0) {
        cur[0] = pos[0] + omega * (cur[0] - pos[0]);
        cur[1] = pos[1] + omega * (cur[1] - pos[1]);
    }
    Xo[2 * node] = cur[0];
    Xo[2 * node + 1] = cur[1];
}

/* Energy (plain ordered sum, weighted) and min det over a sample table. */
void oracle_energy2d(int kind, double delta, const double* X, int64_t ns, const int32_t* gc, const int32_t* gn0,
                     const int32_t* gn1, const double* s0, const double* s1, const double* W, int64_t w_stride,
                     const double* wt, double* energy, double* mindet)
{
    double e = 0.0, m = INFINITY;
    for (int64_t i = 0; i < ns; ++i) {
        double t[4], detA;
        sample_T(X + 2 * (int64_t)gc[i], X + 2 * (int64_t)gn0[i], X + 2 * (int64_t)gn1[i], s0[i], s1[i],
                 W + w_stride * i, t, &detA);
        e += (wt ? wt[i] : 1.0) * mu_value(kind, t, delta);
        if (detA < m) m = detA;
    }
    *energy = e;
    *mindet = m;
}

/* n_sweeps of block-Jacobi; X (2*n_nodes) is updated in place; reports as in
 * the reference (k = report_every <= 0 ? n : report_every). Returns the number
 * of reports written. */
int64_t oracle_run2d(int kind, double delta, double omega, int n_sweeps, int report_every, int64_t n_nodes,
                     double* X, int64_t ndof, const int32_t* dof, const int64_t* off, const int32_t* gc,
                     const int32_t* gn0, const int32_t* gn1, const double* s0, const double* s1,
                     const int32_t* role, const double* W, const double* wt, int64_t ns, const int32_t* es_gc,
                     const int32_t* es_gn0, const int32_t* es_gn1, const double* es_s0, const double* es_s1,
                     const double* es_W, int64_t es_w_stride, const double* es_wt, double* energies,
                     double* mindets)
{
    const patches_t P = {ndof, dof, off, gc, gn0, gn1, s0, s1, role, W, wt};
    double* Xo = (double*)malloc(sizeof(double) * 2 * (size_t)n_nodes);
    if (!Xo) return -1;
    memcpy(Xo, X, sizeof(double) * 2 * (size_t)n_nodes);
    const int k = report_every <= 0 ? n_sweeps : report_every;
    int64_t r = 0;
    for (int s = 0; s < n_sweeps; ++s) {
        for (int64_t d = 0; d < ndof; ++d) update_dof(&P, d, X, Xo, kind, delta, omega);
        memcpy(X, Xo, sizeof(double) * 2 * (size_t)n_nodes);
        if ((s + 1) % k == 0 || s == n_sweeps - 1) {
            oracle_energy2d(kind, delta, X, ns, es_gc, es_gn0, es_gn1, es_s0, es_s1, es_W, es_w_stride, es_wt,
                            &energies[r], &mindets[r]);
            ++r;
        }
    }
    free(Xo);
    return r;
}

/* Per-sample metric (for the golden-vector pin). */
void oracle_metric2d(int kind, double delta, const double* t, double* mu, double* g, double* H)
{
    mu_eval(kind, t, delta, mu, g, H);
}

/* One patch: grad, hess, energy, mindet (for the golden-vector pin). */
void oracle_patch2d(int kind, double delta, const double* X, int32_t P_, const int32_t* gc, const int32_t* gn0,
                    const int32_t* gn1, const double* s0, const double* s1, const double* W, const int32_t* role,
                    double* g, double* h, double* e, double* md, double* step)
{
    const int32_t dof0 = 0;
    const int64_t off[2] = {0, P_};
    const patches_t P = {1, &dof0, off, gc, gn0, gn1, s0, s1, role, W, NULL};
    patch_eval(&P, 0, X, kind, delta, g, h, e, md);
    solve2(h, g, step);
}

/* ======================================================================
 * 3D: mu_cond3 = |T|^2 |cof T|^2 / (9 det^2) - 1 (src/metric.hpp:199-275),
 * its shape+size (+ (det-1)^2) and delta-untangle (det -> Dh) variants
 * (src/metric.hpp:241-262, 877-982).  Value, gradient and the full 9x9
 * Hessian from first/second directional derivatives along the basis
 * directions E_p of vec(T) (row-major), using
 *   s = |T|^2, C = cof T, q = |C|^2, D = det T, F(D) = 1/D^2 or 1/Dh^2,
 *   mu + 1 = s q F / 9,  M(U, V) = d cof / d T (mixed cofactor, bilinear).
 * ====================================================================== */

/* Mixed cofactor M(U,V)_ab = sum eps_acd eps_bef U_ce V_df (symmetric). */
static void mixed_cof(const double U[9], const double V[9], double M[9])
{
    static const int nx[3] = {1, 2, 0}, pv[3] = {2, 0, 1};
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            const int c = nx[a], d = pv[a], e = nx[b], f = pv[b];
            /* eps_acd eps_bef with (c,d) = (a+1, a+2), (e,f) = (b+1, b+2) cyclic:
             * U_ce V_df - U_cf V_de + V_ce U_df - V_cf U_de */
            M[3 * a + b] = U[3 * c + e] * V[3 * d + f] - U[3 * c + f] * V[3 * d + e] + V[3 * c + e] * U[3 * d + f] -
                           V[3 * c + f] * U[3 * d + e];
        }
}

static double det9(const double t[9])
{
    return t[0] * (t[4] * t[8] - t[5] * t[7]) - t[1] * (t[3] * t[8] - t[5] * t[6]) + t[2] * (t[3] * t[7] - t[4] * t[6]);
}

static double mu3_value(int kind, const double t[9], double delta)
{
    double C[9];
    mixed_cof(t, t, C); /* M(T,T) = 2 cof T */
    double s = 0, q = 0;
    for (int i = 0; i < 9; ++i) {
        s += t[i] * t[i];
        q += 0.25 * C[i] * C[i];
    }
    const double D = det9(t);
    double Dd = D;
    if (kind == K_UNTANGLE) Dd = 0.5 * (D + sqrt(D * D + 4.0 * delta * delta));
    double mu = s * q / (9.0 * Dd * Dd) - 1.0;
    if (kind == K_SHAPE_SIZE) mu += (D - 1.0) * (D - 1.0);
    return mu;
}

static void mu3_eval(int kind, const double t[9], double delta, double* mu, double g[9], double H[81])
{
    double C[9], M[9][9], E[9];
    mixed_cof(t, t, C);
    for (int i = 0; i < 9; ++i) C[i] *= 0.5;
    double s = 0, q = 0;
    for (int i = 0; i < 9; ++i) {
        s += t[i] * t[i];
        q += C[i] * C[i];
    }
    const double D = det9(t);
    double F, FD, FDD;
    if (kind == K_UNTANGLE) {
        const double r = sqrt(D * D + 4.0 * delta * delta);
        const double Dh = 0.5 * (D + r), d1 = Dh / r, d2 = 2.0 * delta * delta / (r * r * r);
        F = 1.0 / (Dh * Dh);
        FD = -2.0 * d1 / (Dh * Dh * Dh);
        FDD = 6.0 * d1 * d1 / (Dh * Dh * Dh * Dh) - 2.0 * d2 / (Dh * Dh * Dh);
    } else {
        F = 1.0 / (D * D);
        FD = -2.0 / (D * D * D);
        FDD = 6.0 / (D * D * D * D);
    }
    /* cof(T + eps E) = cof T + eps N(T, E) + eps^2 cof E, with N = mixed_cof:
     * M[p] = d cof [E_p] = N(T, E_p), d2 cof [E_p, E_r] = N(E_p, E_r). */
    for (int p = 0; p < 9; ++p) {
        for (int i = 0; i < 9; ++i) E[i] = (i == p);
        mixed_cof(t, E, M[p]);
    }
    double s1[9], D1[9], q1[9], F1[9];
    for (int p = 0; p < 9; ++p) {
        s1[p] = 2.0 * t[p];
        D1[p] = C[p];
        double acc = 0;
        for (int i = 0; i < 9; ++i) acc += C[i] * M[p][i];
        q1[p] = 2.0 * acc;
        F1[p] = FD * D1[p];
    }
    *mu = s * q * F / 9.0 - 1.0;
    for (int p = 0; p < 9; ++p) g[p] = (s1[p] * q * F + s * q1[p] * F + s * q * F1[p]) / 9.0;
    for (int p = 0; p < 9; ++p)
        for (int r = 0; r < 9; ++r) {
            double Mpr[9];
            for (int i = 0; i < 9; ++i) E[i] = 0.0;
            double Ep[9], Er[9];
            for (int i = 0; i < 9; ++i) {
                Ep[i] = (i == p);
                Er[i] = (i == r);
            }
            mixed_cof(Ep, Er, Mpr);
            double s2 = 2.0 * (p == r);
            double D2 = 0, q2a = 0, q2b = 0;
            for (int i = 0; i < 9; ++i) {
                D2 += Ep[i] * M[r][i];
                q2a += M[p][i] * M[r][i];
                q2b += C[i] * Mpr[i];
            }
            const double q2 = 2.0 * q2a + 2.0 * q2b;
            const double F2 = FDD * D1[p] * D1[r] + FD * D2;
            double h = s2 * q * F + s * q2 * F + s * q * F2 + s1[p] * q1[r] * F + s1[r] * q1[p] * F + s1[p] * q * F1[r] +
                       s1[r] * q * F1[p] + s * q1[p] * F1[r] + s * q1[r] * F1[p];
            H[9 * p + r] = h / 9.0;
            if (kind == K_SHAPE_SIZE) H[9 * p + r] += 2.0 * D1[p] * D1[r] + 2.0 * (D - 1.0) * D2;
        }
    if (kind == K_SHAPE_SIZE) {
        *mu += (D - 1.0) * (D - 1.0);
        for (int p = 0; p < 9; ++p) g[p] += 2.0 * (D - 1.0) * D1[p];
    }
}

/* A[:,k] = s_k (nbr_k - corner), T = A W (row-major 3x3), det A. */
static void sample_T3(const double* c, const double* n0, const double* n1, const double* n2, const double s[3],
                      const double* w, double t[9], double* detA)
{
    const double* nb[3] = {n0, n1, n2};
    double A[9];
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) A[3 * i + k] = s[k] * (nb[k][i] - c[i]);
    *detA = det9(A);
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) {
            double acc = 0;
            for (int j = 0; j < 3; ++j) acc += A[3 * i + j] * w[3 * j + k];
            t[3 * i + k] = acc;
        }
}

static void solve3(const double H[9], const double g[3], double x[3])
{
    const double gn = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
    if (gn < 1e-15) {
        x[0] = x[1] = x[2] = 0.0;
        return;
    }
    const double c00 = H[4] * H[8] - H[5] * H[7], c01 = -(H[3] * H[8] - H[5] * H[6]), c02 = H[3] * H[7] - H[4] * H[6];
    const double det = H[0] * c00 + H[1] * c01 + H[2] * c02;
    const double inv = 1.0 / det;
    const double c10 = -(H[1] * H[8] - H[2] * H[7]), c11 = H[0] * H[8] - H[2] * H[6], c12 = -(H[0] * H[7] - H[1] * H[6]);
    const double c20 = H[1] * H[5] - H[2] * H[4], c21 = -(H[0] * H[5] - H[2] * H[3]), c22 = H[0] * H[4] - H[1] * H[3];
    x[0] = -inv * (c00 * g[0] + c10 * g[1] + c20 * g[2]);
    x[1] = -inv * (c01 * g[0] + c11 * g[1] + c21 * g[2]);
    x[2] = -inv * (c02 * g[0] + c12 * g[1] + c22 * g[2]);
    if (!(isfinite(x[0]) && isfinite(x[1]) && isfinite(x[2]))) {
        const double c = -0.1 / gn;
        for (int k = 0; k < 3; ++k) x[k] = c * g[k];
    }
}

typedef struct {
    int64_t ndof;
    const int32_t* dof;
    const int64_t* off;
    const int32_t* gc;
    const int32_t* gn[3];
    const double* s[3];
    const int32_t* role;
    const double* W; /* [occ*9] */
} patches3_t;

static void patch3_eval(const patches3_t* P, int64_t d, const double* X, int kind, double delta, double g[3],
                        double h[9], double* e, double* md)
{
    for (int k = 0; k < 3; ++k) g[k] = 0.0;
    for (int k = 0; k < 9; ++k) h[k] = 0.0;
    *e = 0.0;
    *md = INFINITY;
    for (int64_t p = P->off[d]; p < P->off[d + 1]; ++p) {
        const double* w = P->W + 9 * p;
        const double sv[3] = {P->s[0][p], P->s[1][p], P->s[2][p]};
        double t[9], detA, mu, gg[9], H[81];
        sample_T3(X + 3 * (int64_t)P->gc[p], X + 3 * (int64_t)P->gn[0][p], X + 3 * (int64_t)P->gn[1][p],
                  X + 3 * (int64_t)P->gn[2][p], sv, w, t, &detA);
        if (detA < *md) *md = detA;
        mu3_eval(kind, t, delta, &mu, gg, H);
        *e += mu;
        const int role = P->role[p];
        if (role < 0) continue;
        double v[3];
        for (int cc = 0; cc < 3; ++cc)
            v[cc] = role == 0 ? -(sv[0] * w[0 * 3 + cc] + sv[1] * w[1 * 3 + cc] + sv[2] * w[2 * 3 + cc])
                              : sv[role - 1] * w[(role - 1) * 3 + cc];
        for (int i = 0; i < 3; ++i) {
            double acc = 0;
            for (int cc = 0; cc < 3; ++cc) acc += gg[3 * i + cc] * v[cc];
            g[i] += acc;
            for (int j = 0; j < 3; ++j) {
                double hh = 0;
                for (int cc = 0; cc < 3; ++cc)
                    for (int c2 = 0; c2 < 3; ++c2) hh += v[cc] * H[9 * (3 * i + cc) + (3 * j + c2)] * v[c2];
                h[3 * i + j] += hh;
            }
        }
    }
}

static void trial3_eval(const patches3_t* P, int64_t d, const double* X, int node, const double tr[3], int kind,
                        double delta, double* e, double* md)
{
    *e = 0.0;
    *md = INFINITY;
    for (int64_t p = P->off[d]; p < P->off[d + 1]; ++p) {
        const int ic = P->gc[p];
        const double* c = ic == node ? tr : X + 3 * (int64_t)ic;
        const double* nb[3];
        for (int k = 0; k < 3; ++k) nb[k] = P->gn[k][p] == node ? tr : X + 3 * (int64_t)P->gn[k][p];
        const double sv[3] = {P->s[0][p], P->s[1][p], P->s[2][p]};
        double t[9], detA;
        sample_T3(c, nb[0], nb[1], nb[2], sv, P->W + 9 * p, t, &detA);
        *e += mu3_value(kind, t, delta);
        if (detA < *md) *md = detA;
    }
}

void oracle_energy3d(int kind, double delta, const double* X, int64_t ns, const int32_t* gc, const int32_t* gn0,
                     const int32_t* gn1, const int32_t* gn2, const double* s0, const double* s1, const double* s2,
                     const double* W, int64_t w_stride, double* energy, double* mindet)
{
    double e = 0.0, m = INFINITY;
    for (int64_t i = 0; i < ns; ++i) {
        const double sv[3] = {s0[i], s1[i], s2[i]};
        double t[9], detA;
        sample_T3(X + 3 * (int64_t)gc[i], X + 3 * (int64_t)gn0[i], X + 3 * (int64_t)gn1[i], X + 3 * (int64_t)gn2[i],
                  sv, W + w_stride * i, t, &detA);
        e += mu3_value(kind, t, delta);
        if (detA < m) m = detA;
    }
    *energy = e;
    *mindet = m;
}

int64_t oracle_run3d(int kind, double delta, double omega, int n_sweeps, int report_every, int64_t n_nodes,
                     double* X, int64_t ndof, const int32_t* dof, const int64_t* off, const int32_t* gc,
                     const int32_t* gn0, const int32_t* gn1, const int32_t* gn2, const double* s0, const double* s1,
                     const double* s2, const int32_t* role, const double* W, int64_t ns, const int32_t* es_gc,
                     const int32_t* es_gn0, const int32_t* es_gn1, const int32_t* es_gn2, const double* es_s0,
                     const double* es_s1, const double* es_s2, const double* es_W, int64_t es_w_stride,
                     double* energies, double* mindets)
{
    const patches3_t P = {ndof, dof, off, gc, {gn0, gn1, gn2}, {s0, s1, s2}, role, W};
    double* Xo = (double*)malloc(sizeof(double) * 3 * (size_t)n_nodes);
    if (!Xo) return -1;
    memcpy(Xo, X, sizeof(double) * 3 * (size_t)n_nodes);
    const int k = report_every <= 0 ? n_sweeps : report_every;
    int64_t r = 0;
    for (int sw = 0; sw < n_sweeps; ++sw) {
        for (int64_t d = 0; d < ndof; ++d) {
            const int node = P.dof[d];
            const double pos[3] = {X[3 * node], X[3 * node + 1], X[3 * node + 2]};
            double g[3], h[9], e0, md0, dl[3];
            patch3_eval(&P, d, X, kind, delta, g, h, &e0, &md0);
            solve3(h, g, dl);
            double alpha = 1.0, cur[3] = {pos[0], pos[1], pos[2]};
            for (int it = 0; it < 10; ++it) {
                const double tr[3] = {pos[0] + alpha * dl[0], pos[1] + alpha * dl[1], pos[2] + alpha * dl[2]};
                double e, md;
                trial3_eval(&P, d, X, node, tr, kind, delta, &e, &md);
                if (isfinite(e) && e <= e0 + 1e-12 && (kind == K_UNTANGLE || md > 0.0)) {
                    for (int q = 0; q < 3; ++q) cur[q] = tr[q];
                    break;
                }
                alpha *= 0.5;
            }
            for (int q = 0; q < 3; ++q) Xo[3 * node + q] = omega != 1.0 ? pos[q] + omega * (cur[q] - pos[q]) : cur[q];
        }
        memcpy(X, Xo, sizeof(double) * 3 * (size_t)n_nodes);
        if ((sw + 1) % k == 0 || sw == n_sweeps - 1) {
            oracle_energy3d(kind, delta, X, ns, es_gc, es_gn0, es_gn1, es_gn2, es_s0, es_s1, es_s2, es_W, es_w_stride,
                            &energies[r], &mindets[r]);
            ++r;
        }
    }
    free(Xo);
    return r;
}

void oracle_metric3d(int kind, double delta, const double* t, double* mu, double* g, double* H)
{
    mu3_eval(kind, t, delta, mu, g, H);
}
