/*
 * CPU FP64 restatement of the near-field EFIE element rule (TEST INFRASTRUCTURE ONLY).
 *
 * The oracle the device near-field fill is checked against. Only tests/ and the CPU legs of
 * bench.py load it; the product path never does.
 *
 * What the reference does (its only executable element routine is the prebuilt CPU
 * `impedance_matrix` of codes/GPU_implementation/seed/functionsExternal.so, called with the
 * argument list of codes/GPU_implementation/seed/compres_single_block_spheres.jl:800-840; the
 * device routines `anal_1divR` / `autoz` are declared without bodies at
 * codes/GPU_implementation/seed/user_impedance_for_julia_cuda.cu:43-44). Black-box runs of that
 * library (tests/golden/make_golden.py) pin the following per triangle pair (Tm, Tn) of an
 * entry, with dc the distance of the two triangle centroids:
 *
 *   - test side: the 4-point degree-3 rule (centroid weight -27/48, points (3/5, 1/5, 1/5)
 *     weight 25/48; Strang & Fix 1973) if dc < Rinteg_f, else the centroid;
 *   - source side: the same 4-point rule if dc < Rinteg_s, else the centroid;
 *   - if dc < Ranal_s, the source integral of G is split into the smooth (exp(-jkR) - 1)/(4 pi R),
 *     taken with the source rule, plus the static 1/(4 pi R) integrated exactly over the source
 *     triangle (the closed-form potentials of Wilton et al., IEEE TAP 1984, written below as
 *     edge-by-edge recursions);
 *   - Tm == Tn (the same triangle) is handled by a separate routine whatever the radii.
 *
 * The first three are reproduced to ~1e-12 relative. The same-triangle routine of the library
 * is not reproduced: its value differs from the exact double integral by a few per cent (its
 * coefficient of k, which every rule integrating constants exactly gets right, is 0.94 of the
 * exact one), so "parity unpinned" holds for same-triangle pairs. Here the same-triangle term
 * is the converged double integral (own method, checked against the closed-form static
 * integral and by refinement):
 *
 *     exp(-jkR)/R = 1/R - (k^2/2) R + (k^4/24) R^3 + rem(R),   rem smooth (C^4)
 *
 *   the 1/R, R and R^3 parts integrated exactly over the source triangle (same recursions),
 *   rem with the 7-point rule, and the outer (test) integral with a rule graded toward the
 *   triangle's edges (three sub-triangles, Gauss-Legendre in both directions with quadratic /
 *   smoothstep substitutions), whose P log P edge behaviour it integrates to ~1e-10.
 *
 * Arrays follow the ccall convention: column-major doubles, 1-based ids stored as doubles.
 */
#include <complex.h>
#include <math.h>
#include <stddef.h>
#include <stdlib.h>

#define NO_PI 3.14159265358979323846
#define NO_GRADED_N 16 /* Gauss-Legendre order per direction of the graded outer rule */

static double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static void cross3(const double *a, const double *b, double *c)
{
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

/* Static potentials of the triangle V at x, for q = -1, 1, 3 (nq = 1: q = -1 only):
   Ip[q] = int_T R^q dS and Y[q] = int_T y R^q dS (R = |x - y|), by the edge recursions
     K_{-1} = log((R+ + l+)/(R- + l-)),  K_q = (l+ R+^q - l- R-^q + q R0^2 K_{q-2}) / (q + 1),
     I_{-1} = sum_i P0_i K_{-1,i} - |d| sum_i beta_i,
     I_q    = (q d^2 I_{q-2} + sum_i P0_i K_{q,i}) / (q + 2),
     int (y - rho0) R^q dS = sum_i u_i K_{q+2,i} / (q + 2),
   with d the height of x over the plane, rho0 its projection, and per edge i its outward
   in-plane normal u_i, the signed distance P0_i of rho0 to the edge line, R0^2 = P0^2 + d^2 and
   the end coordinates l-/l+ along the edge. Returns the triangle area. */
static double potentials(const double *x, const double V[3][3], int nq, double Ip[3], double Y[3][3])
{
    double e1[3], e2[3], nrm[3];
    for (int c = 0; c < 3; ++c) {
        e1[c] = V[1][c] - V[0][c];
        e2[c] = V[2][c] - V[0][c];
    }
    cross3(e1, e2, nrm);
    const double a2 = sqrt(dot3(nrm, nrm));
    double n[3] = {nrm[0] / a2, nrm[1] / a2, nrm[2] / a2};
    double xv[3] = {x[0] - V[0][0], x[1] - V[0][1], x[2] - V[0][2]};
    const double d = dot3(n, xv), ad = fabs(d);
    double rho0[3];
    for (int c = 0; c < 3; ++c) rho0[c] = x[c] - d * n[c];
    double sP[3] = {0, 0, 0}, sB = 0.0, W[3][3] = {{0}};
    for (int i = 0; i < 3; ++i) {
        const double *a = V[i], *b = V[(i + 1) % 3];
        double L[3], lh[3], u[3], ar[3], br[3], xa[3], xb[3];
        for (int c = 0; c < 3; ++c) {
            L[c] = b[c] - a[c];
            ar[c] = a[c] - rho0[c];
            br[c] = b[c] - rho0[c];
            xa[c] = x[c] - a[c];
            xb[c] = x[c] - b[c];
        }
        const double Ll = sqrt(dot3(L, L));
        for (int c = 0; c < 3; ++c) lh[c] = L[c] / Ll;
        cross3(lh, n, u);
        const double lp = dot3(br, lh), lm = dot3(ar, lh), P0 = dot3(ar, u);
        const double R0s = P0 * P0 + d * d;
        const double Rp = sqrt(dot3(xb, xb)), Rm = sqrt(dot3(xa, xa));
        double f = 0.0;
        if (R0s > 1e-28 * Ll * Ll) {
            /* R + l without cancellation: (R + l)(R - l) = R0^2 */
            const double num = lp >= 0 ? Rp + lp : R0s / (Rp - lp);
            const double den = lm >= 0 ? Rm + lm : R0s / (Rm - lm);
            f = log(num / den);
        }
        const double K1 = 0.5 * (lp * Rp - lm * Rm + R0s * f);
        const double Rp2 = Rp * Rp, Rm2 = Rm * Rm;
        const double K3 = 0.25 * (lp * Rp * Rp2 - lm * Rm * Rm2 + 3.0 * R0s * K1);
        const double K5 = (lp * Rp * Rp2 * Rp2 - lm * Rm * Rm2 * Rm2 + 5.0 * R0s * K3) / 6.0;
        if (ad > 0.0)
            sB += atan(P0 * lp / (R0s + ad * Rp)) - atan(P0 * lm / (R0s + ad * Rm));
        sP[0] += P0 * f;
        sP[1] += P0 * K1;
        sP[2] += P0 * K3;
        for (int c = 0; c < 3; ++c) {
            W[0][c] += u[c] * K1;
            W[1][c] += u[c] * K3 / 3.0;
            W[2][c] += u[c] * K5 / 5.0;
        }
    }
    Ip[0] = sP[0] - ad * sB;
    if (nq > 1) {
        Ip[1] = (d * d * Ip[0] + sP[1]) / 3.0;
        Ip[2] = (3.0 * d * d * Ip[1] + sP[2]) / 5.0;
    }
    for (int q = 0; q < nq; ++q)
        for (int c = 0; c < 3; ++c) Y[q][c] = rho0[c] * Ip[q] + W[q][c];
    return 0.5 * a2;
}

/* 4-point degree-3 rule and 7-point degree-5 rule, barycentric */
static const double R4B[4][3] = {{1.0 / 3, 1.0 / 3, 1.0 / 3}, {0.6, 0.2, 0.2}, {0.2, 0.6, 0.2}, {0.2, 0.2, 0.6}};
static const double R4W[4] = {-27.0 / 48.0, 25.0 / 48.0, 25.0 / 48.0, 25.0 / 48.0};

static void rule7(double B[7][3], double W[7])
{
    const double s15 = sqrt(15.0);
    const double a1 = (6.0 - s15) / 21.0, a2 = (6.0 + s15) / 21.0;
    const double w1 = (155.0 - s15) / 1200.0, w2 = (155.0 + s15) / 1200.0;
    B[0][0] = B[0][1] = B[0][2] = 1.0 / 3.0;
    W[0] = 9.0 / 40.0;
    const double A[2] = {a1, a2}, WW[2] = {w1, w2};
    int k = 1;
    for (int g = 0; g < 2; ++g) {
        const double a = A[g], b = 1.0 - 2.0 * a;
        for (int p = 0; p < 3; ++p, ++k) {
            B[k][0] = p == 0 ? b : a;
            B[k][1] = p == 1 ? b : a;
            B[k][2] = p == 2 ? b : a;
            W[k] = WW[g];
        }
    }
}

/* Gauss-Legendre nodes / weights on [0, 1] (Newton on the Legendre recurrence). */
static void gauss_legendre01(int n, double *x, double *w)
{
    for (int i = 0; i < n; ++i) {
        double z = cos(NO_PI * (i + 0.75) / (n + 0.5)), pp = 1.0;
        for (int it = 0; it < 100; ++it) {
            double p1 = 1.0, p2 = 0.0;
            for (int j = 1; j <= n; ++j) {
                const double p3 = p2;
                p2 = p1;
                p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
            }
            pp = n * (z * p1 - p2) / (z * z - 1.0);
            const double dz = p1 / pp;
            z -= dz;
            if (fabs(dz) < 1e-16) break;
        }
        x[i] = 0.5 * (1.0 - z);
        w[i] = 1.0 / ((1.0 - z * z) * pp * pp);
    }
}

/* Outer rule graded toward the edges: 3 n^2 barycentric points, weights summing to 1. For each
   edge (A, B) the sub-triangle (A, B, centroid), p = (1 - s) ((1 - t) A + t B) + s c with
   s = u^2 (dense toward the edge) and t = 3v^2 - 2v^3 (dense toward both ends). */
static int graded_rule(int n, double *B, double *W)
{
    double *gx = malloc(sizeof(double) * n), *gw = malloc(sizeof(double) * n);
    gauss_legendre01(n, gx, gw);
    const double Vb[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    int k = 0;
    double tot = 0.0;
    for (int e = 0; e < 3; ++e) {
        const double *A = Vb[e], *Bv = Vb[(e + 1) % 3];
        for (int i = 0; i < n; ++i) {
            const double u = gx[i], s = u * u, ws = 2.0 * u * gw[i];
            for (int j = 0; j < n; ++j) {
                const double v = gx[j], t = 3 * v * v - 2 * v * v * v, wt = (6 * v - 6 * v * v) * gw[j];
                for (int c = 0; c < 3; ++c)
                    B[3 * k + c] = (1 - s) * ((1 - t) * A[c] + t * Bv[c]) + s / 3.0;
                W[k] = ws * wt * (1 - s);
                tot += W[k];
                ++k;
            }
        }
    }
    for (int i = 0; i < k; ++i) W[i] /= tot;
    free(gx);
    free(gw);
    return k;
}

/* exp(-jkR)/R - 1/R + (k^2/2) R - (k^4/24) R^3 (smooth; limit -jk at R = 0) */
static double complex smooth_rem(double R, double k)
{
    const double x = k * R;
    double re;
    if (x < 0.6) {
        const double x2 = x * x;
        re = k * x2 * x2 * x *
             (-1.0 / 720 + x2 * (1.0 / 40320 + x2 * (-1.0 / 3628800 + x2 * (1.0 / 479001600 - x2 / 87178291200.0))));
    } else {
        re = (cos(x) - 1.0 + 0.5 * x * x - x * x * x * x / 24.0) / R;
    }
    const double im = x < 1e-8 ? -k : -sin(x) / R;
    return re + I * im;
}

static void tri_vertices(int t, const double *vertex, const double *topol, double V[3][3])
{
    for (int c = 0; c < 3; ++c) {
        const int v = (int)topol[3 * (size_t)t + c] - 1;
        for (int d = 0; d < 3; ++d) V[c][d] = vertex[3 * (size_t)v + d];
    }
}

/* Same-triangle moments (normalised by the area squared, G = exp(-jkR)/(4 pi R)):
   m[0] = <G>, m[1..3] = <x G>, m[4..6] = <y G>, m[7] = <x.y G> over T x T. */
void oracle_self_moments(double complex *m, const double V[3][3], double k, int n)
{
    const double C = 1.0 / (4.0 * NO_PI);
    double *B = malloc(sizeof(double) * 9 * n * n), *W = malloc(sizeof(double) * 3 * n * n);
    const int np = graded_rule(n, B, W);
    double B7[7][3], W7[7], Y7[7][3];
    rule7(B7, W7);
    for (int q = 0; q < 7; ++q)
        for (int d = 0; d < 3; ++d) Y7[q][d] = B7[q][0] * V[0][d] + B7[q][1] * V[1][d] + B7[q][2] * V[2][d];
    for (int i = 0; i < 8; ++i) m[i] = 0.0;
    for (int p = 0; p < np; ++p) {
        double x[3];
        for (int d = 0; d < 3; ++d) x[d] = B[3 * p] * V[0][d] + B[3 * p + 1] * V[1][d] + B[3 * p + 2] * V[2][d];
        double Iq[3], Yq[3][3];
        const double A = potentials(x, V, 3, Iq, Yq);
        double complex J1 = C * (Iq[0] - 0.5 * k * k * Iq[1] + k * k * k * k / 24.0 * Iq[2]) / A;
        double complex Jy[3];
        for (int d = 0; d < 3; ++d)
            Jy[d] = C * (Yq[0][d] - 0.5 * k * k * Yq[1][d] + k * k * k * k / 24.0 * Yq[2][d]) / A;
        for (int q = 0; q < 7; ++q) {
            double dd[3] = {x[0] - Y7[q][0], x[1] - Y7[q][1], x[2] - Y7[q][2]};
            const double complex r = C * W7[q] * smooth_rem(sqrt(dot3(dd, dd)), k);
            J1 += r;
            for (int d = 0; d < 3; ++d) Jy[d] += r * Y7[q][d];
        }
        m[0] += W[p] * J1;
        for (int d = 0; d < 3; ++d) {
            m[1 + d] += W[p] * x[d] * J1;
            m[4 + d] += W[p] * Jy[d];
        }
        m[7] += W[p] * (x[0] * Jy[0] + x[1] * Jy[1] + x[2] * Jy[2]);
    }
    free(B);
    free(W);
}

typedef struct {
    int n;
    double P[7][3], w[7];
} pts_t;

static void side_points(int four, int q_far, int t, const double *vertex, const double *topol,
                        const double *cent, pts_t *o)
{
    double V[3][3];
    if (four) {
        tri_vertices(t, vertex, topol, V);
        o->n = 4;
        for (int p = 0; p < 4; ++p) {
            o->w[p] = R4W[p];
            for (int d = 0; d < 3; ++d)
                o->P[p][d] = R4B[p][0] * V[0][d] + R4B[p][1] * V[1][d] + R4B[p][2] * V[2][d];
        }
    } else if (q_far == 7) {
        double B7[7][3];
        tri_vertices(t, vertex, topol, V);
        rule7(B7, o->w);
        o->n = 7;
        for (int p = 0; p < 7; ++p)
            for (int d = 0; d < 3; ++d)
                o->P[p][d] = B7[p][0] * V[0][d] + B7[p][1] * V[1][d] + B7[p][2] * V[2][d];
    } else {
        o->n = 1;
        o->w[0] = 1.0;
        for (int d = 0; d < 3; ++d) o->P[0][d] = cent[3 * (size_t)t + d];
    }
}

/* Near-field fill Z(r1, r2) (column-major n_r1 x n_r2). rs / ra / rf = Rinteg_s, Ranal_s,
   Rinteg_f; q_far = rule of a side outside its radius (1 = centroid, as the reference; 7).
   n_self = graded-rule order of the same-triangle term (0: default). Returns 0 or -1. */
int oracle_fill_near(double *Zr, double *Zi, double k, double eta, double rs, double ra, double rf,
                     int q_far, int n_self, const double *r1, const double *r2, int n_r1, int n_r2,
                     const double *vertex, const double *topol, const double *edges,
                     const double *ln, const double *cent, int n_edges, int n_tri)
{
    if (q_far != 1 && q_far != 7) return -1;
    if (n_self <= 0) n_self = NO_GRADED_N;
    const double C = 1.0 / (4.0 * NO_PI);
    /* same-triangle moments, computed on first use */
    double complex *mom = calloc((size_t)n_tri * 8, sizeof(double complex));
    char *have = calloc((size_t)n_tri, 1);
    for (int j = 0; j < n_r2; ++j) {
        const int nb = (int)r2[j] - 1;
        if (nb < 0 || nb >= n_edges) goto bad;
        for (int i = 0; i < n_r1; ++i) {
            const int ma = (int)r1[i] - 1;
            if (ma < 0 || ma >= n_edges) goto bad;
            const double la = ln[ma], lb = ln[nb];
            double complex z = 0.0;
            for (int a = 0; a < 2; ++a) {
                const double sa = a == 0 ? 1.0 : -1.0;
                const int ta = (int)edges[4 * (size_t)ma + a] - 1, oa = (int)edges[4 * (size_t)ma + 2 + a] - 1;
                const double *va = vertex + 3 * (size_t)oa;
                for (int b = 0; b < 2; ++b) {
                    const double sb = b == 0 ? 1.0 : -1.0;
                    const int tb = (int)edges[4 * (size_t)nb + b] - 1, ob = (int)edges[4 * (size_t)nb + 2 + b] - 1;
                    const double *vb = vertex + 3 * (size_t)ob;
                    if (ta == tb) {
                        if (!have[ta]) {
                            double V[3][3];
                            tri_vertices(ta, vertex, topol, V);
                            oracle_self_moments(mom + 8 * (size_t)ta, V, k, n_self);
                            have[ta] = 1;
                        }
                        const double complex *M = mom + 8 * (size_t)ta;
                        const double complex P = sa * sb *
                            (M[7] - (vb[0] * M[1] + vb[1] * M[2] + vb[2] * M[3]) -
                             (va[0] * M[4] + va[1] * M[5] + va[2] * M[6]) + dot3(va, vb) * M[0]);
                        z += I * k * eta * (la * lb / 4.0) * P - I * (eta / k) * sa * sb * la * lb * M[0];
                        continue;
                    }
                    double dcv[3];
                    for (int d = 0; d < 3; ++d) dcv[d] = cent[3 * (size_t)ta + d] - cent[3 * (size_t)tb + d];
                    const double dc = sqrt(dot3(dcv, dcv));
                    pts_t pt, ps;
                    side_points(dc < rf, q_far, ta, vertex, topol, cent, &pt);
                    side_points(dc < rs, q_far, tb, vertex, topol, cent, &ps);
                    const int anal = dc < ra;
                    double VS[3][3];
                    if (anal) tri_vertices(tb, vertex, topol, VS);
                    for (int p = 0; p < pt.n; ++p) {
                        const double *x = pt.P[p];
                        double rho_a[3] = {sa * (x[0] - va[0]), sa * (x[1] - va[1]), sa * (x[2] - va[2])};
                        double complex Sg = 0.0, Sr[3] = {0, 0, 0};
                        for (int q = 0; q < ps.n; ++q) {
                            const double *y = ps.P[q];
                            double dd[3] = {x[0] - y[0], x[1] - y[1], x[2] - y[2]};
                            const double R = sqrt(dot3(dd, dd));
                            const double complex g = (cexp(-I * k * R) - (anal ? 1.0 : 0.0)) * C / R;
                            Sg += ps.w[q] * g;
                            for (int d = 0; d < 3; ++d) Sr[d] += ps.w[q] * g * sb * (y[d] - vb[d]);
                        }
                        if (anal) {
                            double Iq[3], Yq[3][3];
                            const double A = potentials(x, VS, 1, Iq, Yq);
                            Sg += C * Iq[0] / A;
                            for (int d = 0; d < 3; ++d) Sr[d] += C * sb * (Yq[0][d] - vb[d] * Iq[0]) / A;
                        }
                        z += pt.w[p] * (I * k * eta * (la * lb / 4.0) *
                                            (rho_a[0] * Sr[0] + rho_a[1] * Sr[1] + rho_a[2] * Sr[2]) -
                                        I * (eta / k) * sa * sb * la * lb * Sg);
                    }
                }
            }
            z = -z;
            Zr[i + (size_t)j * n_r1] = creal(z);
            Zi[i + (size_t)j * n_r1] = cimag(z);
        }
    }
    free(mom);
    free(have);
    return 0;
bad:
    free(mom);
    free(have);
    return -1;
}

/* Same-triangle moments of triangle t (0-based) for tests: m as 16 doubles (re, im pairs). */
int oracle_self_moments_tri(double *out, int t, double k, int n, const double *vertex,
                            const double *topol)
{
    double V[3][3];
    double complex m[8];
    tri_vertices(t, vertex, topol, V);
    oracle_self_moments(m, V, k, n > 0 ? n : NO_GRADED_N);
    for (int i = 0; i < 8; ++i) {
        out[2 * i] = creal(m[i]);
        out[2 * i + 1] = cimag(m[i]);
    }
    return 0;
}
