// Near-field EFIE element rule on the device (FP64, one thread per entry).
//
// The reference's element routine (the CPU `impedance_matrix` of functionsExternal.so, called as
// at compres_single_block_spheres.jl:800-840; its device counterparts `anal_1divR` / `autoz` are
// declared without bodies at user_impedance_for_julia_cuda.cu:43-44) switches per triangle pair
// (Tm, Tn), by the distance dc of the two triangle centroids:
//   - test side:   4-point degree-3 rule if dc < Rinteg_f, else the centroid;
//   - source side: 4-point degree-3 rule if dc < Rinteg_s, else the centroid;
//   - dc < Ranal_s: the source integral of G = exp(-jkR)/(4 pi R) is the smooth
//     (exp(-jkR) - 1)/(4 pi R) by the source rule plus the static 1/(4 pi R) integrated exactly
//     over the source triangle;
//   - Tm == Tn: a separate same-triangle term, whatever the radii.
// The first three are reproduced exactly (the closed-form static potentials of the source
// triangle, Wilton et al. IEEE TAP 1984, as edge recursions). The same-triangle term is the
// converged double integral instead of the library's approximation: exp(-jkR)/R is split into
// 1/R - (k^2/2) R + (k^4/24) R^3 (integrated exactly over the source triangle by the same
// recursions) plus a C^4 remainder (7-point rule), and the outer integral uses a rule graded
// toward the triangle's edges (3 x 16 x 16 points). Its eight moments per triangle
// (<G>, <x G>, <y G>, <x.y G>) are computed once per triangle and reused by every RWG pair that
// shares the triangle.
//
// Every entry is independent: one thread per entry, the CTA's 256 entries column-major within a
// job (consecutive rows -> coalesced stores). Mesh arrays are read in the reference layout.
#include <cmath>
#include <mutex>
#include <vector>

#include "engine_internal.cuh"

namespace pskel {

constexpr int kGradedN = 16;
constexpr int kGradedPts = 3 * kGradedN * kGradedN;  // 768
constexpr int kNearThreads = 256;

__constant__ double c_graded[kGradedPts * 4];  // barycentric (3) + weight, weights sum to 1
__constant__ double c_rule7[7 * 4];
__constant__ double c_rule4[4 * 4];

namespace {

// Gauss-Legendre nodes and weights on [0, 1] (Newton on the three-term recurrence).
void gauss_legendre01(int n, double *x, double *w) {
    const double pi = 3.14159265358979323846;
    for (int i = 0; i < n; ++i) {
        double z = std::cos(pi * (i + 0.75) / (n + 0.5)), pp = 1.0;
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
            if (std::fabs(dz) < 1e-16) break;
        }
        x[i] = 0.5 * (1.0 - z);
        w[i] = 1.0 / ((1.0 - z * z) * pp * pp);
    }
}

// Rules uploaded once per device: the graded outer rule of the same-triangle term (for each edge
// (A, B) the sub-triangle (A, B, centroid); p = (1 - s)((1 - t) A + t B) + s c, s = u^2 toward
// the edge, t = 3v^2 - 2v^3 toward both ends), the 7-point degree-5 rule (Radon; Dunavant n = 5)
// and the 4-point degree-3 rule (Strang & Fix).
int upload_rules() {
    static std::mutex mu;
    static unsigned long long done = 0;  // bit per device
    int dev = 0;
    PSKEL_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    if (dev < 64 && (done >> dev) & 1ull) return PSKEL_OK;
    std::vector<double> g(kGradedPts * 4);
    double gx[kGradedN], gw[kGradedN];
    gauss_legendre01(kGradedN, gx, gw);
    const double Vb[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    double tot = 0.0;
    int k = 0;
    for (int e = 0; e < 3; ++e) {
        const double *A = Vb[e], *B = Vb[(e + 1) % 3];
        for (int i = 0; i < kGradedN; ++i) {
            const double u = gx[i], s = u * u, ws = 2.0 * u * gw[i];
            for (int j = 0; j < kGradedN; ++j) {
                const double v = gx[j], t = 3 * v * v - 2 * v * v * v, wt = (6 * v - 6 * v * v) * gw[j];
                for (int c = 0; c < 3; ++c) g[4 * k + c] = (1 - s) * ((1 - t) * A[c] + t * B[c]) + s / 3.0;
                g[4 * k + 3] = ws * wt * (1 - s);
                tot += g[4 * k + 3];
                ++k;
            }
        }
    }
    for (int i = 0; i < kGradedPts; ++i) g[4 * i + 3] /= tot;
    double r7[28];
    {
        const double s15 = std::sqrt(15.0);
        const double a[2] = {(6.0 - s15) / 21.0, (6.0 + s15) / 21.0};
        const double w[2] = {(155.0 - s15) / 1200.0, (155.0 + s15) / 1200.0};
        r7[0] = r7[1] = r7[2] = 1.0 / 3.0;
        r7[3] = 9.0 / 40.0;
        int q = 1;
        for (int gi = 0; gi < 2; ++gi)
            for (int p = 0; p < 3; ++p, ++q) {
                const double b = 1.0 - 2.0 * a[gi];
                r7[4 * q + 0] = p == 0 ? b : a[gi];
                r7[4 * q + 1] = p == 1 ? b : a[gi];
                r7[4 * q + 2] = p == 2 ? b : a[gi];
                r7[4 * q + 3] = w[gi];
            }
    }
    const double r4[16] = {1.0 / 3, 1.0 / 3, 1.0 / 3, -27.0 / 48.0, 0.6, 0.2, 0.2, 25.0 / 48.0,
                           0.2, 0.6, 0.2, 25.0 / 48.0, 0.2, 0.2, 0.6, 25.0 / 48.0};
    PSKEL_CUDA(cudaMemcpyToSymbol(c_graded, g.data(), sizeof(double) * g.size()));
    PSKEL_CUDA(cudaMemcpyToSymbol(c_rule7, r7, sizeof(r7)));
    PSKEL_CUDA(cudaMemcpyToSymbol(c_rule4, r4, sizeof(r4)));
    if (dev < 64) done |= 1ull << dev;
    return PSKEL_OK;
}

__device__ __forceinline__ double dot3(const double *a, const double *b) {
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
__device__ __forceinline__ void cross3(const double *a, const double *b, double *c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

// Static potentials of triangle V at x for q = -1 (and 1, 3 when NQ = 3):
// Ip[q] = int R^q dS, Y[q] = int y R^q dS, by the edge recursions
//   K_-1 = log((R+ + l+)/(R- + l-)), K_q = (l+ R+^q - l- R-^q + q R0^2 K_{q-2}) / (q + 1),
//   I_-1 = sum P0 K_-1 - |d| sum beta, I_q = (q d^2 I_{q-2} + sum P0 K_q) / (q + 2),
//   int (y - rho0) R^q dS = sum u K_{q+2} / (q + 2).
// Returns the area.
template <int NQ>
__device__ double potentials(const double *x, const double (*V)[3], double *Ip, double (*Y)[3]) {
    double e1[3], e2[3], nrm[3];
    for (int c = 0; c < 3; ++c) {
        e1[c] = V[1][c] - V[0][c];
        e2[c] = V[2][c] - V[0][c];
    }
    cross3(e1, e2, nrm);
    const double a2 = sqrt(dot3(nrm, nrm));
    const double n[3] = {nrm[0] / a2, nrm[1] / a2, nrm[2] / a2};
    const double xv[3] = {x[0] - V[0][0], x[1] - V[0][1], x[2] - V[0][2]};
    const double d = dot3(n, xv), ad = fabs(d);
    double rho0[3];
    for (int c = 0; c < 3; ++c) rho0[c] = x[c] - d * n[c];
    double sP[3] = {0, 0, 0}, sB = 0.0, W[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll 1
    for (int i = 0; i < 3; ++i) {
        const double *a = V[i], *b = V[i == 2 ? 0 : i + 1];
        double L[3], ar[3], br[3], xa[3], xb[3];
        for (int c = 0; c < 3; ++c) {
            L[c] = b[c] - a[c];
            ar[c] = a[c] - rho0[c];
            br[c] = b[c] - rho0[c];
            xa[c] = x[c] - a[c];
            xb[c] = x[c] - b[c];
        }
        const double Ll = sqrt(dot3(L, L));
        const double lh[3] = {L[0] / Ll, L[1] / Ll, L[2] / Ll};
        double u[3];
        cross3(lh, n, u);
        const double lp = dot3(br, lh), lm = dot3(ar, lh), P0 = dot3(ar, u);
        const double R0s = P0 * P0 + d * d;
        const double Rp = sqrt(dot3(xb, xb)), Rm = sqrt(dot3(xa, xa));
        double f = 0.0;
        if (R0s > 1e-28 * Ll * Ll) {
            const double num = lp >= 0 ? Rp + lp : R0s / (Rp - lp);
            const double den = lm >= 0 ? Rm + lm : R0s / (Rm - lm);
            f = log(num / den);
        }
        const double K1 = 0.5 * (lp * Rp - lm * Rm + R0s * f);
        if (ad > 0.0) sB += atan(P0 * lp / (R0s + ad * Rp)) - atan(P0 * lm / (R0s + ad * Rm));
        sP[0] += P0 * f;
        for (int c = 0; c < 3; ++c) W[0][c] += u[c] * K1;
        if (NQ > 1) {
            const double Rp2 = Rp * Rp, Rm2 = Rm * Rm;
            const double K3 = 0.25 * (lp * Rp * Rp2 - lm * Rm * Rm2 + 3.0 * R0s * K1);
            const double K5 = (lp * Rp * Rp2 * Rp2 - lm * Rm * Rm2 * Rm2 + 5.0 * R0s * K3) / 6.0;
            sP[1] += P0 * K1;
            sP[2] += P0 * K3;
            for (int c = 0; c < 3; ++c) {
                W[1][c] += u[c] * K3 / 3.0;
                W[2][c] += u[c] * K5 / 5.0;
            }
        }
    }
    Ip[0] = sP[0] - ad * sB;
    if (NQ > 1) {
        Ip[1] = (d * d * Ip[0] + sP[1]) / 3.0;
        Ip[2] = (3.0 * d * d * Ip[1] + sP[2]) / 5.0;
    }
    for (int q = 0; q < NQ; ++q)
        for (int c = 0; c < 3; ++c) Y[q][c] = rho0[c] * Ip[q] + W[q][c];
    return 0.5 * a2;
}

// exp(-jkR)/R - 1/R + (k^2/2) R - (k^4/24) R^3, limit -jk at R = 0.
__device__ __forceinline__ double2 smooth_rem(double R, double k) {
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
    return make_double2(re, im);
}

__device__ __forceinline__ bool load_tri(int t, const double *vertex, const double *topol, int nv,
                                         double (*V)[3]) {
    for (int c = 0; c < 3; ++c) {
        const double vd = topol[3 * (size_t)t + c];
        if (!(vd >= 1.0 && vd <= (double)nv)) return false;
        const int v = (int)vd - 1;
        for (int d = 0; d < 3; ++d) V[c][d] = vertex[3 * (size_t)v + d];
    }
    return true;
}

// One CTA per triangle: its eight same-triangle moments (normalised by the area squared),
// <G>, <x G> (3), <y G> (3), <x.y G>, as double2 (re, im) at mom[8 t ...].
// tri_of: NULL -> triangle blockIdx.x; else triangle = edges[4 rwg + side] - 1 for
// rwg = rwg_list[blockIdx.x / 2], side = blockIdx.x % 2.
__global__ void __launch_bounds__(kNearThreads)
self_moments_kernel(const double *__restrict__ vertex, const double *__restrict__ topol,
                    const double *__restrict__ edges, int ne, int nt, int nv,
                    const int *__restrict__ rwg_list, double k, double2 *__restrict__ mom,
                    int *flags) {
    __shared__ double red[kNearThreads / 32][16];
    int t = blockIdx.x;
    if (rwg_list) {
        const int e = rwg_list[blockIdx.x >> 1];
        if (e < 0 || e >= ne) {
            if (threadIdx.x == 0) atomicOr(flags, 2);
            return;
        }
        const double td = edges[4 * (size_t)e + (blockIdx.x & 1)];
        if (!(td >= 1.0 && td <= (double)nt)) {
            if (threadIdx.x == 0) atomicOr(flags, 4);
            return;
        }
        t = (int)td - 1;
    }
    double V[3][3];
    if (!load_tri(t, vertex, topol, nv, V)) {
        if (threadIdx.x == 0) atomicOr(flags, 4);
        return;
    }
    const double C = 0.07957747154594767;  // 1 / (4 pi)
    double Y7[7][3];
    for (int q = 0; q < 7; ++q)
        for (int d = 0; d < 3; ++d)
            Y7[q][d] = c_rule7[4 * q] * V[0][d] + c_rule7[4 * q + 1] * V[1][d] + c_rule7[4 * q + 2] * V[2][d];
    double acc[16];
    for (int i = 0; i < 16; ++i) acc[i] = 0.0;
    const double k2 = 0.5 * k * k, k4 = k * k * k * k / 24.0;
    for (int p = threadIdx.x; p < kGradedPts; p += kNearThreads) {
        const double b0 = c_graded[4 * p], b1 = c_graded[4 * p + 1], b2 = c_graded[4 * p + 2];
        const double w = c_graded[4 * p + 3];
        double x[3];
        for (int d = 0; d < 3; ++d) x[d] = b0 * V[0][d] + b1 * V[1][d] + b2 * V[2][d];
        double Ip[3], Yq[3][3];
        const double A = potentials<3>(x, V, Ip, Yq);
        double j1r = C * (Ip[0] - k2 * Ip[1] + k4 * Ip[2]) / A, j1i = 0.0;
        double jyr[3], jyi[3] = {0, 0, 0};
        for (int d = 0; d < 3; ++d) jyr[d] = C * (Yq[0][d] - k2 * Yq[1][d] + k4 * Yq[2][d]) / A;
        for (int q = 0; q < 7; ++q) {
            const double dd[3] = {x[0] - Y7[q][0], x[1] - Y7[q][1], x[2] - Y7[q][2]};
            const double2 r = smooth_rem(sqrt(dot3(dd, dd)), k);
            const double cw = C * c_rule7[4 * q + 3];
            j1r += cw * r.x;
            j1i += cw * r.y;
            for (int d = 0; d < 3; ++d) {
                jyr[d] += cw * r.x * Y7[q][d];
                jyi[d] += cw * r.y * Y7[q][d];
            }
        }
        acc[0] += w * j1r;
        acc[1] += w * j1i;
        for (int d = 0; d < 3; ++d) {
            acc[2 + 2 * d] += w * x[d] * j1r;
            acc[3 + 2 * d] += w * x[d] * j1i;
            acc[8 + 2 * d] += w * jyr[d];
            acc[9 + 2 * d] += w * jyi[d];
        }
        acc[14] += w * (x[0] * jyr[0] + x[1] * jyr[1] + x[2] * jyr[2]);
        acc[15] += w * (x[0] * jyi[0] + x[1] * jyi[1] + x[2] * jyi[2]);
    }
    for (int i = 0; i < 16; ++i)
        for (int o = 16; o; o >>= 1) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0)
        for (int i = 0; i < 16; ++i) red[wid][i] = acc[i];
    __syncthreads();
    if (threadIdx.x < 16) {
        double s = 0.0;
        for (int q = 0; q < kNearThreads / 32; ++q) s += red[q][threadIdx.x];
        reinterpret_cast<double *>(mom + 8 * (size_t)t)[threadIdx.x] = s;
    }
}

struct NearArgs {
    double k, eta, rs, ra, rf;
    int q_far;
    int patch;  // 1: only entries with a triangle pair inside a radius or a same-triangle pair
};

// Does entry (m, n) have a same-triangle pair or a pair with centroid distance below a radius?
__device__ __forceinline__ bool entry_is_near(int m, int n, const double *__restrict__ edges,
                                              const double *__restrict__ cent, int nt, double rmax) {
    for (int a = 0; a < 2; ++a) {
        const double tad = edges[4 * (size_t)m + a];
        if (!(tad >= 1.0 && tad <= (double)nt)) return true;  // let the full path report it
        const double *ca = cent + 3 * ((size_t)tad - 1);
        for (int b = 0; b < 2; ++b) {
            const double tbd = edges[4 * (size_t)n + b];
            if (!(tbd >= 1.0 && tbd <= (double)nt) || tad == tbd) return true;
            const double *cb = cent + 3 * ((size_t)tbd - 1);
            const double dcv[3] = {ca[0] - cb[0], ca[1] - cb[1], ca[2] - cb[2]};
            if (sqrt(dot3(dcv, dcv)) < rmax) return true;  // as near_entry computes dc
        }
    }
    return false;
}

// Rule of one side: 0 = centroid, 1 = the 4-point rule, 2 = the 7-point rule. Points are formed
// when used (no per-side point arrays: fewer registers, more resident warps).
__device__ __forceinline__ int side_rule(bool four, int q_far) { return four ? 1 : (q_far == 7 ? 2 : 0); }
__device__ __forceinline__ int rule_points(int rule) { return rule == 1 ? 4 : (rule == 2 ? 7 : 1); }
__device__ __forceinline__ double rule_point(int rule, int p, const double (*V)[3], const double *cen,
                                             double *x) {
    if (rule == 0) {
        x[0] = cen[0];
        x[1] = cen[1];
        x[2] = cen[2];
        return 1.0;
    }
    const double *b = rule == 1 ? c_rule4 + 4 * p : c_rule7 + 4 * p;
    for (int d = 0; d < 3; ++d) x[d] = b[0] * V[0][d] + b[1] * V[1][d] + b[2] * V[2][d];
    return b[3];
}

// One entry Z(m, n). Returns false on an out-of-range id inside the mesh arrays.
__device__ bool near_entry(int m, int n, const double *__restrict__ vertex,
                           const double *__restrict__ topol, const double *__restrict__ edges,
                           const double *__restrict__ ln, const double *__restrict__ cent, int nt,
                           int nv, const NearArgs &a, const double2 *__restrict__ mom,
                           double2 *out) {
    const double C = 0.07957747154594767;  // 1 / (4 pi)
    const double lm = ln[m], lnn = ln[n];
    const double cdiv = a.eta / a.k * lm * lnn;      // (eta / k) l_m l_n
    const double cvec = a.k * a.eta * lm * lnn / 4.0;  // k eta l_m l_n / 4
    double zr = 0.0, zi = 0.0;
#pragma unroll 1
    for (int sa_i = 0; sa_i < 2; ++sa_i) {
        const double sa = sa_i == 0 ? 1.0 : -1.0;
        const double tad = edges[4 * (size_t)m + sa_i], oad = edges[4 * (size_t)m + 2 + sa_i];
        if (!(tad >= 1.0 && tad <= (double)nt && oad >= 1.0 && oad <= (double)nv)) return false;
        const int ta = (int)tad - 1;
        const double *va = vertex + 3 * ((size_t)oad - 1);
        double VT[3][3];
        if (!load_tri(ta, vertex, topol, nv, VT)) return false;
#pragma unroll 1
        for (int sb_i = 0; sb_i < 2; ++sb_i) {
            const double sb = sb_i == 0 ? 1.0 : -1.0;
            const double tbd = edges[4 * (size_t)n + sb_i], obd = edges[4 * (size_t)n + 2 + sb_i];
            if (!(tbd >= 1.0 && tbd <= (double)nt && obd >= 1.0 && obd <= (double)nv)) return false;
            const int tb = (int)tbd - 1;
            const double *vb = vertex + 3 * ((size_t)obd - 1);
            const double ss = sa * sb;
            if (ta == tb) {
                const double2 *M = mom + 8 * (size_t)ta;
                // P = <rho_a . rho_b G> = sa sb (<x.y G> - vb.<x G> - va.<y G> + va.vb <G>)
                double p_re = M[7].x - (vb[0] * M[1].x + vb[1] * M[2].x + vb[2] * M[3].x) -
                            (va[0] * M[4].x + va[1] * M[5].x + va[2] * M[6].x) + dot3(va, vb) * M[0].x;
                double p_im = M[7].y - (vb[0] * M[1].y + vb[1] * M[2].y + vb[2] * M[3].y) -
                            (va[0] * M[4].y + va[1] * M[5].y + va[2] * M[6].y) + dot3(va, vb) * M[0].y;
                p_re *= ss;
                p_im *= ss;
                // z += j cvec P - j cdiv ss <G>
                zr += -cvec * p_im + cdiv * ss * M[0].y;
                zi += cvec * p_re - cdiv * ss * M[0].x;
                continue;
            }
            const double *ca = cent + 3 * (size_t)ta, *cb = cent + 3 * (size_t)tb;
            const double dcv[3] = {ca[0] - cb[0], ca[1] - cb[1], ca[2] - cb[2]};
            const double dc = sqrt(dot3(dcv, dcv));
            double VS[3][3];
            if (!load_tri(tb, vertex, topol, nv, VS)) return false;
            const int rt = side_rule(dc < a.rf, a.q_far), rsr = side_rule(dc < a.rs, a.q_far);
            const int ntp = rule_points(rt), nsp = rule_points(rsr);
            const bool anal = dc < a.ra;
#pragma unroll 1
            for (int p = 0; p < ntp; ++p) {
                double x[3];
                const double wtp = rule_point(rt, p, VT, ca, x);
                const double rho_a[3] = {sa * (x[0] - va[0]), sa * (x[1] - va[1]), sa * (x[2] - va[2])};
                double sgr = 0.0, sgi = 0.0, srr[3] = {0, 0, 0}, sri[3] = {0, 0, 0};
#pragma unroll 1
                for (int q = 0; q < nsp; ++q) {
                    double y[3];
                    const double wsq = rule_point(rsr, q, VS, cb, y);
                    const double dd[3] = {x[0] - y[0], x[1] - y[1], x[2] - y[2]};
                    const double R = sqrt(dot3(dd, dd));
                    double s, c;
                    sincos(a.k * R, &s, &c);
                    const double f = wsq * C / R;
                    const double gr = (c - (anal ? 1.0 : 0.0)) * f, gi = -s * f;
                    sgr += gr;
                    sgi += gi;
                    for (int d = 0; d < 3; ++d) {
                        const double rb = sb * (y[d] - vb[d]);
                        srr[d] += gr * rb;
                        sri[d] += gi * rb;
                    }
                }
                if (anal) {
                    double Ip[1], Yq[1][3];
                    const double A = potentials<1>(x, VS, Ip, Yq);
                    sgr += C * Ip[0] / A;
                    for (int d = 0; d < 3; ++d) srr[d] += C * sb * (Yq[0][d] - vb[d] * Ip[0]) / A;
                }
                const double dr = dot3(rho_a, srr), di = dot3(rho_a, sri);
                // z += w_p (j cvec (rho_a . S_r) - j cdiv ss S_g)
                zr += wtp * (-cvec * di + cdiv * ss * sgi);
                zi += wtp * (cvec * dr - cdiv * ss * sgr);
            }
        }
    }
    *out = make_double2(-zr, -zi);
    return true;
}

__global__ void __launch_bounds__(kNearThreads, 2)
near_fill_kernel(const double *__restrict__ vertex, const double *__restrict__ topol,
                 const double *__restrict__ edges, const double *__restrict__ ln,
                 const double *__restrict__ cent, int ne, int nt, int nv,
                 const FillJob *__restrict__ jobs, const long long *__restrict__ prefix, int njobs,
                 NearArgs a, const double2 *__restrict__ mom, int *flags) {
    const long long tile = blockIdx.x;
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {  // last job with prefix[j] <= tile
        const int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= tile) lo = mid; else hi = mid - 1;
    }
    const FillJob job = jobs[lo];
    const long long e = (tile - prefix[lo]) * kNearThreads + threadIdx.x;
    if (e >= (long long)job.nr * job.nc) return;
    const int i = (int)(e % job.nr), j = (int)(e / job.nr);
    const int m = job.rows[i], n = job.cols[j];
    if (m < 0 || m >= ne || n < 0 || n >= ne) {
        atomicOr(flags, 2);
        return;
    }
    if (a.patch && !entry_is_near(m, n, edges, cent, nt, fmax(a.rs, fmax(a.ra, a.rf)))) return;
    double2 z;
    if (!near_entry(m, n, vertex, topol, edges, ln, cent, nt, nv, a, mom, &z)) {
        atomicOr(flags, 4);
        z = make_double2(0.0, 0.0);
    }
    double2 *o = static_cast<double2 *>(job.out);
    if (job.trans) o[j + (size_t)i * job.ld] = z; else o[i + (size_t)j * job.ld] = z;
}

}  // namespace

int near_fill_jobs(const DevMesh &mesh, const NearRadii &r, double k, double eta,
                   const std::vector<FillJob> &jobs, DevBuf &scratch, DevBuf &mom, int *d_flags,
                   cudaStream_t stream, bool all_triangles, bool patch) {
    PSKEL_TRY(upload_rules());
    if (jobs.empty()) return PSKEL_OK;
    std::vector<long long> prefix(jobs.size() + 1, 0);
    for (size_t i = 0; i < jobs.size(); ++i)
        prefix[i + 1] = prefix[i] + ((long long)jobs[i].nr * jobs[i].nc + kNearThreads - 1) / kNearThreads;
    if (prefix.back() == 0) return PSKEL_OK;
    if (prefix.back() > 0x7fffffffLL) {
        set_error(PSKEL_ERR_ARG, "near fill: %lld tiles (limit 2^31 - 1)", prefix.back());
        return PSKEL_ERR_ARG;
    }
    const size_t jb = (sizeof(FillJob) * jobs.size() + 255) & ~size_t(255);
    PSKEL_TRY(scratch.reserve(jb + sizeof(long long) * prefix.size()));
    FillJob *d_jobs = scratch.as<FillJob>();
    long long *d_prefix = reinterpret_cast<long long *>(scratch.as<char>() + jb);
    PSKEL_CUDA(cudaMemcpyAsync(d_jobs, jobs.data(), sizeof(FillJob) * jobs.size(),
                               cudaMemcpyHostToDevice, stream));
    PSKEL_CUDA(cudaMemcpyAsync(d_prefix, prefix.data(), sizeof(long long) * prefix.size(),
                               cudaMemcpyHostToDevice, stream));
    PSKEL_TRY(mom.reserve(sizeof(double2) * 8 * (size_t)mesh.nt));
    // same-triangle moments: every triangle, or the triangles of the rows of each job (a
    // same-triangle pair's triangle belongs to its test RWG)
    if (all_triangles) {
        self_moments_kernel<<<mesh.nt, kNearThreads, 0, stream>>>(
            mesh.vertex.as<double>(), mesh.topol.as<double>(), mesh.edges.as<double>(), mesh.ne,
            mesh.nt, mesh.nv, nullptr, k, mom.as<double2>(), d_flags);
        PSKEL_LAUNCHED(1);
    } else {
        for (const FillJob &j : jobs) {
            if ((long long)j.nr * j.nc == 0) continue;
            self_moments_kernel<<<2 * j.nr, kNearThreads, 0, stream>>>(
                mesh.vertex.as<double>(), mesh.topol.as<double>(), mesh.edges.as<double>(), mesh.ne,
                mesh.nt, mesh.nv, j.rows, k, mom.as<double2>(), d_flags);
            PSKEL_LAUNCHED(1);
        }
    }
    NearArgs a{k, eta, r.rinteg_s, r.ranal_s, r.rinteg_f, r.q_far, patch ? 1 : 0};
    near_fill_kernel<<<(unsigned)prefix.back(), kNearThreads, 0, stream>>>(
        mesh.vertex.as<double>(), mesh.topol.as<double>(), mesh.edges.as<double>(),
        mesh.ln.as<double>(), mesh.cent.as<double>(), mesh.ne, mesh.nt, mesh.nv, d_jobs, d_prefix,
        (int)jobs.size(), a, mom.as<double2>(), d_flags);
    PSKEL_LAUNCHED(1);
    return PSKEL_OK;
}

}  // namespace pskel

extern "C" int pskel_fill_near_device(pskel_ctx *c, const int *rows_dev, int nr,
                                      const int *cols_dev, int nc, pskel_c128 *Z_dev, int ld,
                                      double rinteg_s, double ranal_s, double rinteg_f, int q_far) {
    using namespace pskel;
    if (!c) {
        set_error(PSKEL_ERR_ARG, "fill_near: null context");
        return PSKEL_ERR_ARG;
    }
    PSKEL_CUDA(cudaSetDevice(c->device));
    if (!c->have_mesh) {
        set_error(PSKEL_ERR_STATE, "fill_near: no mesh uploaded");
        return PSKEL_ERR_STATE;
    }
    if (nr < 0 || nc < 0 || ld < nr || (q_far != 1 && q_far != 7) || !(rinteg_s >= 0) ||
        !(ranal_s >= 0) || !(rinteg_f >= 0) || ((size_t)nr * nc > 0 && (!rows_dev || !cols_dev || !Z_dev))) {
        set_error(PSKEL_ERR_ARG, "fill_near: nr=%d nc=%d ld=%d q_far=%d radii %g %g %g", nr, nc, ld,
                  q_far, rinteg_s, ranal_s, rinteg_f);
        return PSKEL_ERR_ARG;
    }
    if ((size_t)nr * nc == 0) return PSKEL_OK;
    NearRadii r;
    r.rinteg_s = rinteg_s;
    r.ranal_s = ranal_s;
    r.rinteg_f = rinteg_f;
    r.q_far = q_far;
    std::vector<FillJob> jobs{FillJob{rows_dev, cols_dev, Z_dev, nr, nc, ld, 0}};
    return near_fill_jobs(c->mesh, r, c->em.k, c->em.eta, jobs, c->near_jobs, c->near_mom,
                          c->flags.as<int>(), c->stream, false, false);
}
