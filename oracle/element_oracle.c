/*
 * CPU FP64 restatement of the RWG/EFIE impedance-element integral (TEST INFRASTRUCTURE ONLY).
 *
 * This file is the oracle the CUDA fill kernels are checked against. Only tests/, the smoke
 * check and the CPU-baseline leg of bench.py load it; the product path never does.
 *
 * Reference behaviour it restates:
 *   - the device element routine `impedance_matrix_single_element2` is declared but has no
 *     body in codes/GPU_implementation/seed/user_impedance_for_julia_cuda.cu:178-214; the
 *     only executable element routine is the prebuilt CPU `impedance_matrix` in
 *     codes/GPU_implementation/seed/functionsExternal.so, called with the argument list of
 *     codes/GPU_implementation/seed/compres_single_block_spheres.jl:800-840.
 *   - For a triangle pair farther apart than the integration radii, that routine evaluates a
 *     one-point (centroid) rule per triangle. The formula below reproduces it to ~1e-15
 *     relative (pinned by tests/golden fixtures generated from the shipped library):
 *
 *       Z_mn = - sum_{Tm in {T+,T-}} sum_{Tn in {T+,T-}} sum_p sum_q w_p w_q G(R_pq) *
 *              [ j k eta (l_m l_n / 4) rho_m(r_p).rho_n(r_q) - j (eta/k) s_m s_n l_m l_n ]
 *
 *     with G(R) = exp(-j k R) / (4 pi R), rho = s (r - v_opp), s = +1 on T+ and -1 on T-
 *     (standard RWG/EFIE Galerkin form, Rao-Wilton-Glisson, IEEE TAP 1982).
 *   - q = 7 is the 7-point degree-5 triangle rule (Radon 1948; Dunavant 1985 table, n=5):
 *     centroid weight 9/40, points (a,a,1-2a) with a = (6 -+ sqrt 15)/21 and weights
 *     (155 -+ sqrt 15)/1200. It has no counterpart in the reference and is validated by
 *     self-convergence against a refined composite rule.
 *
 * Arrays follow the ccall convention: column-major doubles, 1-based ids stored as doubles.
 */
#include <complex.h>
#include <math.h>
#include <stddef.h>

#define ORACLE_PI 3.14159265358979323846

typedef struct {
    int n;
    double a[7], b[7], c[7], w[7];
} tri_rule;

static void make_rule(int q, tri_rule *r)
{
    if (q == 1) {
        r->n = 1;
        r->a[0] = r->b[0] = r->c[0] = 1.0 / 3.0;
        r->w[0] = 1.0;
        return;
    }
    const double s15 = sqrt(15.0);
    const double a1 = (6.0 - s15) / 21.0, a2 = (6.0 + s15) / 21.0;
    const double w1 = (155.0 - s15) / 1200.0, w2 = (155.0 + s15) / 1200.0;
    r->n = 7;
    r->a[0] = r->b[0] = r->c[0] = 1.0 / 3.0;
    r->w[0] = 9.0 / 40.0;
    const double A[2] = {a1, a2}, W[2] = {w1, w2};
    int k = 1;
    for (int g = 0; g < 2; ++g) {
        const double a = A[g], b = 1.0 - 2.0 * a;
        double bc[3][3] = {{b, a, a}, {a, b, a}, {a, a, b}};
        for (int p = 0; p < 3; ++p, ++k) {
            r->a[k] = bc[p][0];
            r->b[k] = bc[p][1];
            r->c[k] = bc[p][2];
            r->w[k] = W[g];
        }
    }
}

/* quadrature points of triangle t (0-based); q == 1 uses the stored centroid so that the
   arithmetic is the same as the shipped routine's centroid path. */
static void tri_points(const tri_rule *r, int t, const double *vertex, const double *topol,
                       const double *cent, double pts[7][3])
{
    if (r->n == 1) {
        for (int d = 0; d < 3; ++d) pts[0][d] = cent[3 * (size_t)t + d];
        return;
    }
    const int v1 = (int)topol[3 * (size_t)t + 0] - 1;
    const int v2 = (int)topol[3 * (size_t)t + 1] - 1;
    const int v3 = (int)topol[3 * (size_t)t + 2] - 1;
    for (int p = 0; p < r->n; ++p)
        for (int d = 0; d < 3; ++d)
            pts[p][d] = r->a[p] * vertex[3 * (size_t)v1 + d] + r->b[p] * vertex[3 * (size_t)v2 + d] +
                        r->c[p] * vertex[3 * (size_t)v3 + d];
}

static double complex element(int m, int n, double k, double eta, const tri_rule *rt,
                              const tri_rule *rs, const double *vertex, const double *topol,
                              const double *edges, const double *ln, const double *cent)
{
    double complex acc = 0.0;
    const double lm = ln[m], lnn = ln[n];
    for (int a = 0; a < 2; ++a) {
        const double sa = a == 0 ? 1.0 : -1.0;
        const int ta = (int)edges[4 * (size_t)m + a] - 1;
        const int va = (int)edges[4 * (size_t)m + 2 + a] - 1;
        double pa[7][3];
        tri_points(rt, ta, vertex, topol, cent, pa);
        for (int b = 0; b < 2; ++b) {
            const double sb = b == 0 ? 1.0 : -1.0;
            const int tb = (int)edges[4 * (size_t)n + b] - 1;
            const int vb = (int)edges[4 * (size_t)n + 2 + b] - 1;
            double pb[7][3];
            tri_points(rs, tb, vertex, topol, cent, pb);
            for (int p = 0; p < rt->n; ++p) {
                double rho_a[3];
                for (int d = 0; d < 3; ++d) rho_a[d] = sa * (pa[p][d] - vertex[3 * (size_t)va + d]);
                for (int q = 0; q < rs->n; ++q) {
                    double rho_b[3], dd[3];
                    for (int d = 0; d < 3; ++d) {
                        rho_b[d] = sb * (pb[q][d] - vertex[3 * (size_t)vb + d]);
                        dd[d] = pa[p][d] - pb[q][d];
                    }
                    const double R = sqrt(dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2]);
                    const double complex G = cexp(-I * k * R) / (4.0 * ORACLE_PI * R);
                    const double dot = rho_a[0] * rho_b[0] + rho_a[1] * rho_b[1] + rho_a[2] * rho_b[2];
                    const double complex kern =
                        I * k * eta * (lm * lnn / 4.0) * dot - I * (eta / k) * sa * sb * lm * lnn;
                    acc += rt->w[p] * rs->w[q] * G * kern;
                }
            }
        }
    }
    return -acc;
}

/* Fill Z(r1, r2) (column-major, n_r1 x n_r2) with q_test / q_src points per triangle
   (1 or 7). r1/r2 hold 1-based RWG ids as doubles. Returns 0, or -1 on a bad argument. */
int oracle_fill(double *Zr, double *Zi, double k, double eta, int q_test, int q_src,
                const double *r1, const double *r2, int n_r1, int n_r2, const double *vertex,
                const double *topol, const double *edges, const double *ln, const double *cent,
                int n_edges)
{
    if ((q_test != 1 && q_test != 7) || (q_src != 1 && q_src != 7)) return -1;
    tri_rule rt, rs;
    make_rule(q_test, &rt);
    make_rule(q_src, &rs);
    for (int j = 0; j < n_r2; ++j) {
        const int n = (int)r2[j] - 1;
        if (n < 0 || n >= n_edges) return -1;
        for (int i = 0; i < n_r1; ++i) {
            const int m = (int)r1[i] - 1;
            if (m < 0 || m >= n_edges) return -1;
            const double complex z =
                element(m, n, k, eta, &rt, &rs, vertex, topol, edges, ln, cent);
            Zr[i + (size_t)j * n_r1] = creal(z);
            Zi[i + (size_t)j * n_r1] = cimag(z);
        }
    }
    return 0;
}

/* Composite centroid rule on 4^level congruent sub-triangles per side: an independent,
   slowly converging reference used only to validate the 7-point rule. */
static void sub_centroids(const double v[3][3], int level, double *out, int *count)
{
    if (level == 0) {
        for (int d = 0; d < 3; ++d) out[3 * (*count) + d] = (v[0][d] + v[1][d] + v[2][d]) / 3.0;
        (*count)++;
        return;
    }
    double m01[3], m12[3], m20[3];
    for (int d = 0; d < 3; ++d) {
        m01[d] = 0.5 * (v[0][d] + v[1][d]);
        m12[d] = 0.5 * (v[1][d] + v[2][d]);
        m20[d] = 0.5 * (v[2][d] + v[0][d]);
    }
    double t[4][3][3];
    for (int d = 0; d < 3; ++d) {
        t[0][0][d] = v[0][d]; t[0][1][d] = m01[d]; t[0][2][d] = m20[d];
        t[1][0][d] = m01[d]; t[1][1][d] = v[1][d]; t[1][2][d] = m12[d];
        t[2][0][d] = m20[d]; t[2][1][d] = m12[d]; t[2][2][d] = v[2][d];
        t[3][0][d] = m01[d]; t[3][1][d] = m12[d]; t[3][2][d] = m20[d];
    }
    for (int s = 0; s < 4; ++s) sub_centroids(t[s], level - 1, out, count);
}

int oracle_element_composite(double *zr, double *zi, double k, double eta, int m1, int n1,
                             int level, const double *vertex, const double *topol,
                             const double *edges, const double *ln, double *work)
{
    /* work must hold 2 * 3 * 4^level doubles */
    const int m = m1 - 1, n = n1 - 1;
    int npts = 1;
    for (int l = 0; l < level; ++l) npts *= 4;
    double *pa = work, *pb = work + 3 * (size_t)npts;
    const double w = 1.0 / npts;
    double complex acc = 0.0;
    for (int a = 0; a < 2; ++a) {
        const double sa = a == 0 ? 1.0 : -1.0;
        const int ta = (int)edges[4 * (size_t)m + a] - 1, va = (int)edges[4 * (size_t)m + 2 + a] - 1;
        double v[3][3];
        for (int c = 0; c < 3; ++c)
            for (int d = 0; d < 3; ++d) v[c][d] = vertex[3 * ((size_t)topol[3 * (size_t)ta + c] - 1) + d];
        int cnt = 0;
        sub_centroids(v, level, pa, &cnt);
        for (int b = 0; b < 2; ++b) {
            const double sb = b == 0 ? 1.0 : -1.0;
            const int tb = (int)edges[4 * (size_t)n + b] - 1, vb = (int)edges[4 * (size_t)n + 2 + b] - 1;
            double u[3][3];
            for (int c = 0; c < 3; ++c)
                for (int d = 0; d < 3; ++d) u[c][d] = vertex[3 * ((size_t)topol[3 * (size_t)tb + c] - 1) + d];
            int cnt2 = 0;
            sub_centroids(u, level, pb, &cnt2);
            for (int p = 0; p < npts; ++p)
                for (int q = 0; q < npts; ++q) {
                    double ra[3], rb[3], dd[3];
                    for (int d = 0; d < 3; ++d) {
                        ra[d] = sa * (pa[3 * p + d] - vertex[3 * (size_t)va + d]);
                        rb[d] = sb * (pb[3 * q + d] - vertex[3 * (size_t)vb + d]);
                        dd[d] = pa[3 * p + d] - pb[3 * q + d];
                    }
                    const double R = sqrt(dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2]);
                    const double complex G = cexp(-I * k * R) / (4.0 * ORACLE_PI * R);
                    const double dot = ra[0] * rb[0] + ra[1] * rb[1] + ra[2] * rb[2];
                    acc += w * w * G *
                           (I * k * eta * (ln[m] * ln[n] / 4.0) * dot - I * (eta / k) * sa * sb * ln[m] * ln[n]);
                }
        }
    }
    *zr = creal(-acc);
    *zi = cimag(-acc);
    return 0;
}
