// RWG/EFIE element fill: batched Z(rows, cols) sub-blocks for arbitrary id lists.
//
// Replaces the one-thread-per-element kernels impedance_matrix_compute_elbyel2/3
// (codes/GPU_implementation/seed/user_impedance_for_julia_cuda.cu:256-439), whose per-element
// body impedance_matrix_single_element2 (declared at :178-214) is absent from the reference
// source. The arithmetic restates the reference CPU routine's far-field rule (centroid rule per
// triangle, Q = 1) and adds the 7-point rule (Q = 7):
//
//   Z_mn = eta/(4 pi) * sum_{p in test points} sum_{q in source points} A_pq (sin kR + j cos kR)/R
//   A_pq = d_p e_q / k - k u_p . v_q          (record fields, see pskel_internal.cuh)
//
// Precision: c128 evaluates everything in FP64. c64 keeps the geometry in FP64 - the point
// differences, R and the phase reduced to a fraction of a wavelength, f = R/lambda - rint(R/lambda)
// - and does the rest in FP32 (sin/cos of 2 pi f with sincospif, 1/R, the kernel products and
// the accumulation). A pure-FP32 distance has an absolute error of ~1e-7 lambda at a few
// wavelengths, i.e. a phase error of ~1e-6 rad per point pair, which the cancellation between
// the four triangle-pair terms of a far RWG interaction amplifies to ~1e-5 relative error in
// Z; FP64 geometry brings the c64 fill to ~1e-6 (the FP64 pipe of B200 runs at half the FP32
// rate, so the extra dozen FP64 operations per point pair are affordable).
//
// Design (B200): the kernel is bound by the FP64 (c128) or FP32/FP64/MUFU (c64) pipes, not by
// memory. A CTA owns a TM x TN tile of one job; the TM test and TN source records are gathered
// once into shared memory (coalesced; positions as doubles, vectors/charges in the arithmetic
// type, odd strides), each
// thread then evaluates (2Q)^2 point pairs for its entry with the test point held in registers
// and the source points broadcast from shared memory. With SPLIT > 1 the source points of one
// entry are spread over SPLIT adjacent lanes and combined with warp shuffles (used for small
// fills where there are too few entries to fill the GPU). The grid is persistent: a multiple of
// the SM count, striding over the global tile list of all jobs (no atomics, no waits).
#include <cmath>

#include "pskel_internal.cuh"

namespace pskel {

template <typename T> struct Cplx;
template <> struct Cplx<double> { using type = double2; };
template <> struct Cplx<float> { using type = float2; };

// c64: R and the phase in turns t = R k / (2 pi) in FP64, the fraction f = t - rint(t) in
// [-1/2, 1/2] rounded to FP32, then sin(2 pi f), cos(2 pi f) = sincospif(2 f) in FP32.
__device__ __forceinline__ void green_sincos_mixed(double R, double kturn, float *s, float *c) {
    const double t = R * kturn;
    const float f = (float)(t - rint(t));
    sincospif(2.0f * f, s, c);
}

__device__ __forceinline__ int find_job(const int *__restrict__ prefix, int njobs, int tile) {
    int lo = 0, hi = njobs;  // prefix[lo] <= tile < prefix[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(prefix + mid) <= tile) lo = mid; else hi = mid;
    }
    return lo;
}

// Minimum resident CTAs per SM requested from the register allocator.
template <typename T> struct FillOcc { static constexpr int value = sizeof(T) == 8 ? 2 : 3; };

// Records are read from the FP64 record array; positions are staged in shared memory as G
// (double) and the weighted RWG vectors/charges as T.
template <typename T, int Q, int TM, int TN, int SPLIT, bool GATED = false>
__global__ void __launch_bounds__(TM *TN *SPLIT, FillOcc<T>::value)
    fill_kernel(const double *__restrict__ rec_t, const double *__restrict__ rec_s,
                const FillJob *__restrict__ jobs, const int *__restrict__ tile_prefix, int njobs,
                int total_tiles, T k, T kinv, double kphase, T scale, double r_near2, int *flags,
                const int *const *__restrict__ gates) {
    constexpr int NP = 2 * Q;
    constexpr int RS = (7 * NP) | 1;
    constexpr int PS = (3 * NP) | 1;  // staged position stride (doubles)
    constexpr int VS = (4 * NP) | 1;  // staged vector/charge stride (T)
    constexpr int NT = TM * TN * SPLIT;
    using C2 = typename Cplx<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *p_t = reinterpret_cast<double *>(smem_raw);  // TM x PS positions
    double *p_s = p_t + TM * PS;                          // TN x PS
    T *v_t = reinterpret_cast<T *>(p_s + TN * PS);        // TM x VS
    T *v_s = v_t + TM * VS;                               // TN x VS

    const int tid = threadIdx.x;
    const int ls = tid % SPLIT;
    const int e = tid / SPLIT;
    const int il = e % TM;
    const int jl = e / TM;

    for (int tile = blockIdx.x; tile < total_tiles; tile += gridDim.x) {
        const int jb = find_job(tile_prefix, njobs, tile);
        if constexpr (GATED) {
            if (*gates[jb] == 0) continue;  // uniform over the CTA
        }
        const FillJob job = jobs[jb];
        const int local = tile - tile_prefix[jb];
        const int tiles_r = (job.nr + TM - 1) / TM;
        const int i0 = (local % tiles_r) * TM;
        const int j0 = (local / tiles_r) * TN;

        for (int idx = tid; idx < TM * 7 * NP; idx += NT) {
            const int r = idx / (7 * NP), f = idx - r * (7 * NP);
            const int row = i0 + r;
            const double v = row < job.nr ? rec_t[(size_t)job.rows[row] * RS + f] : 0.0;
            if (f < 3 * NP) p_t[r * PS + f] = v; else v_t[r * VS + f - 3 * NP] = (T)v;
        }
        for (int idx = tid; idx < TN * 7 * NP; idx += NT) {
            const int r = idx / (7 * NP), f = idx - r * (7 * NP);
            const int col = j0 + r;
            const double v = col < job.nc ? rec_s[(size_t)job.cols[col] * RS + f] : 0.0;
            if (f < 3 * NP) p_s[r * PS + f] = v; else v_s[r * VS + f - 3 * NP] = (T)v;
        }
        __syncthreads();

        const int i = i0 + il, j = j0 + jl;
        const bool live = i < job.nr && j < job.nc;
        T re = 0, im = 0;
        if (live) {
            const double *pt = p_t + il * PS;
            const double *ps = p_s + jl * PS;
            const T *vt = v_t + il * VS;
            const T *vs = v_s + jl * VS;
            if (r_near2 > 0.0 && ls == 0) {
                // point 0 of each side is the triangle centroid (Q = 1 and Q = 7 rules)
                bool near = false;
#pragma unroll
                for (int a = 0; a < 2; ++a)
#pragma unroll
                    for (int b = 0; b < 2; ++b) {
                        const double dx = pt[a * Q] - ps[b * Q];
                        const double dy = pt[NP + a * Q] - ps[NP + b * Q];
                        const double dz = pt[2 * NP + a * Q] - ps[2 * NP + b * Q];
                        near |= dx * dx + dy * dy + dz * dz < r_near2;
                    }
                if (near) atomicOr(flags, 1);
            }
#pragma unroll 1
            for (int p = 0; p < NP; ++p) {
                const double xp = pt[p], yp = pt[NP + p], zp = pt[2 * NP + p];
                const T ux = k * vt[p], uy = k * vt[NP + p], uz = k * vt[2 * NP + p];
                const T dp = kinv * vt[3 * NP + p];
#pragma unroll 2
                for (int q = ls; q < NP; q += SPLIT) {
                    const double dx = xp - ps[q], dy = yp - ps[NP + q], dz = zp - ps[2 * NP + q];
                    const double R2 = fma(dx, dx, fma(dy, dy, dz * dz));
                    T sn, cs, rinv;
                    if constexpr (sizeof(T) == 8) {
                        rinv = rsqrt(R2);
                        sincospi(R2 * rinv * kphase, &sn, &cs);
                    } else {
                        // 1/R from the FP32 reciprocal square root; R refined in FP64 by one
                        // Newton step from it, so that the phase keeps FP64 accuracy.
                        const float y = rsqrtf((float)R2);
                        const double R0 = R2 * (double)y;
                        const double R = fma(0.5 * (double)y, fma(-R0, R0, R2), R0);
                        green_sincos_mixed(R, kphase, &sn, &cs);
                        rinv = y;
                    }
                    const T A = fma(dp, vs[3 * NP + q],
                                    -fma(ux, vs[q], fma(uy, vs[NP + q], uz * vs[2 * NP + q])));
                    const T t = A * rinv;
                    re = fma(t, sn, re);
                    im = fma(t, cs, im);
                }
            }
        }
        if (SPLIT > 1) {
#pragma unroll
            for (int o = 1; o < SPLIT; o <<= 1) {
                re += __shfl_xor_sync(0xffffffffu, re, o);
                im += __shfl_xor_sync(0xffffffffu, im, o);
            }
        }
        if (live && ls == 0) {
            C2 z;
            z.x = scale * re;
            z.y = scale * im;
            C2 *out = reinterpret_cast<C2 *>(job.out);
            if (!job.trans) out[i + (size_t)j * job.ld] = z;
            else out[j + (size_t)i * job.ld] = z;
        }
        __syncthreads();
    }
}

// ===================================================================== default fill kernel
// Sin and cos of the phase, evaluated without a library call: the phase t (in wavelengths, FP64)
// is split as t = q/4 + g with q = rint(4 t) (the integer lands in the low mantissa word of
// 4 t + 1.5 * 2^52, so no conversion instruction is needed) and |g| <= 1/8, then
// sin/cos(2 pi g) come from their Taylor series about 0 (coefficients (-1)^k / n!), truncated
// where the first omitted term is below half an ulp at |2 pi g| = pi/4 (FP32: theta^9 / theta^10,
// FP64: theta^17 / theta^16), and a rotation by q quarter turns gives sin/cos(2 pi t).
__host__ __device__ constexpr double inv_fact(int n) { return n <= 1 ? 1.0 : inv_fact(n - 1) / n; }

__device__ __forceinline__ void rotate_quadrant(int q, float sn, float cs, float *s, float *c) {
    float a = (q & 1) ? cs : sn;
    float b = (q & 1) ? sn : cs;
    *s = (q & 2) ? -a : a;
    *c = ((q + 1) & 2) ? -b : b;
}
__device__ __forceinline__ void rotate_quadrant(int q, double sn, double cs, double *s, double *c) {
    double a = (q & 1) ? cs : sn;
    double b = (q & 1) ? sn : cs;
    *s = (q & 2) ? -a : a;
    *c = ((q + 1) & 2) ? -b : b;
}

__device__ __forceinline__ void sincos_2pi(float g, int q, float *s, float *c) {
    const float th = g * 6.28318530717958647692f;
    const float t2 = th * th;
    float ps = fmaf(t2, (float)inv_fact(9), -(float)inv_fact(7));
    ps = fmaf(t2, ps, (float)inv_fact(5));
    ps = fmaf(t2, ps, -(float)inv_fact(3));
    const float sn = fmaf(th * t2, ps, th);
    float pc = fmaf(t2, -(float)inv_fact(10), (float)inv_fact(8));
    pc = fmaf(t2, pc, -(float)inv_fact(6));
    pc = fmaf(t2, pc, (float)inv_fact(4));
    pc = fmaf(t2, pc, -0.5f);
    const float cs = fmaf(t2, pc, 1.0f);
    rotate_quadrant(q, sn, cs, s, c);
}

// sin/cos(2 pi g) for |g| <= 1/4 turn (|theta| <= pi/2), no quadrant rotation, as polynomials in
// s = g^2 on [0, 1/16]: sin(2 pi g) = g P(s), cos(2 pi g) = 1 + s Q(s), P and Q of degree 4 that
// interpolate sin(2 pi g) / g and (cos(2 pi g) - 1) / g^2 at the five Chebyshev nodes of the
// interval (near-minimax: 7e-9 and 9e-10 before rounding, below FP32's own rounding; evaluated
// in FP32 both stay within 1.3 ulp of 1, as the degree-5 and -6 Taylor series in g did). Used
// with a half-turn reduction t = n/2 + g, where sin and cos of 2 pi t both take the sign (-1)^n.
__device__ __forceinline__ void sincos_2pi_half(float g, float *s, float *c) {
    const float t2 = g * g;
    float ps = fmaf(t2, 39.759827f, -76.58117f);
    ps = fmaf(t2, ps, 81.60248f);
    ps = fmaf(t2, ps, -41.341682f);
    ps = fmaf(t2, ps, 6.2831855f);
    *s = g * ps;
    float pc = fmaf(t2, -25.218163f, 60.17904f);
    pc = fmaf(t2, pc, -85.45536f);
    pc = fmaf(t2, pc, 64.939384f);
    pc = fmaf(t2, pc, -19.739208f);
    *c = fmaf(t2, pc, 1.0f);
}

__device__ __forceinline__ void sincos_2pi(double g, int q, double *s, double *c) {
    const double th = g * 6.28318530717958647692;
    const double t2 = th * th;
    double ps = fma(t2, inv_fact(17), -inv_fact(15));
    ps = fma(t2, ps, inv_fact(13));
    ps = fma(t2, ps, -inv_fact(11));
    ps = fma(t2, ps, inv_fact(9));
    ps = fma(t2, ps, -inv_fact(7));
    ps = fma(t2, ps, inv_fact(5));
    ps = fma(t2, ps, -inv_fact(3));
    const double sn = fma(th * t2, ps, th);
    double pc = fma(t2, inv_fact(16), -inv_fact(14));
    pc = fma(t2, pc, inv_fact(12));
    pc = fma(t2, pc, -inv_fact(10));
    pc = fma(t2, pc, inv_fact(8));
    pc = fma(t2, pc, -inv_fact(6));
    pc = fma(t2, pc, inv_fact(4));
    pc = fma(t2, pc, -0.5);
    const double cs = fma(t2, pc, 1.0);
    rotate_quadrant(q, sn, cs, s, c);
}

// t (wavelengths) -> (g, q) with t = q/4 + g, |g| <= 1/8
__device__ __forceinline__ double split_quarter(double t, int *q) {
    const double M = 6755399441055744.0;  // 1.5 * 2^52
    const double tm = fma(t, 4.0, M);
    *q = __double2loint(tm);
    return fma(tm - M, -0.25, t);
}

template <typename T> struct Vec4;
template <> struct Vec4<float> { using type = float4; };
template <> struct Vec4<double> { using type = double4; };
template <typename T> struct Fill2Occ { static constexpr int value = sizeof(T) == 8 ? 2 : 3; };

// Two rows per thread: thread (il, jl) computes entries (i0 + il, j) and (i0 + il + TM/2, j),
// so every source point read from shared memory serves two entries. Source points are staged
// as {x, y} (double2), z (double), {ux, uy, uz, e} (T4); test points field-major per row with
// odd strides. Persistent grid over the tile list of all jobs, like fill_kernel.
template <typename T, int Q, int TM, int TN, bool GATED = false>
__global__ void __launch_bounds__(TM / 2 * TN, Fill2Occ<T>::value)
    fill2_kernel(const double *__restrict__ rec_t, const double *__restrict__ rec_s,
                 const FillJob *__restrict__ jobs, const int *__restrict__ tile_prefix,
                 int njobs, int total_tiles, T k, T kinv, double kturn, T scale,
                 double r_near2, int *flags, const int *const *__restrict__ gates) {
    constexpr int NP = 2 * Q;
    constexpr int RS = (7 * NP) | 1;
    constexpr int PS = (3 * NP) | 1;
    constexpr int VS = (4 * NP) | 1;
    constexpr int HALF = TM / 2;
    constexpr int NT = HALF * TN;
    using C2 = typename Cplx<T>::type;
    using T4 = typename Vec4<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *s_xy = reinterpret_cast<double2 *>(smem_raw);         // TN x NP
    double *s_z = reinterpret_cast<double *>(s_xy + TN * NP);        // TN x NP
    T4 *s_v = reinterpret_cast<T4 *>(s_z + TN * NP);                 // TN x NP
    double *p_t = reinterpret_cast<double *>(s_v + TN * NP);         // TM x PS
    T *v_t = reinterpret_cast<T *>(p_t + TM * PS);                   // TM x VS

    const int tid = threadIdx.x;
    const int il = tid % HALF;
    const int jl = tid / HALF;

    for (int tile = blockIdx.x; tile < total_tiles; tile += gridDim.x) {
        const int jb = find_job(tile_prefix, njobs, tile);
        if constexpr (GATED) {
            if (*gates[jb] == 0) continue;  // uniform over the CTA
        }
        const FillJob job = jobs[jb];
        const int local = tile - tile_prefix[jb];
        const int tiles_r = (job.nr + TM - 1) / TM;
        const int i0 = (local % tiles_r) * TM;
        const int j0 = (local / tiles_r) * TN;

        for (int idx = tid; idx < TM * 7 * NP; idx += NT) {
            const int r = idx / (7 * NP), f = idx - r * (7 * NP);
            const int row = i0 + r;
            const double v = row < job.nr ? rec_t[(size_t)job.rows[row] * RS + f] : 0.0;
            if (f < 3 * NP) p_t[r * PS + f] = v; else v_t[r * VS + f - 3 * NP] = (T)v;
        }
        for (int idx = tid; idx < TN * NP; idx += NT) {
            const int c = idx / NP, q = idx - c * NP;
            const int col = j0 + c;
            const double *src = rec_s + (size_t)(col < job.nc ? job.cols[col] : 0) * RS;
            const bool ok = col < job.nc;
            s_xy[idx] = make_double2(ok ? src[q] : 0.0, ok ? src[NP + q] : 0.0);
            s_z[idx] = ok ? src[2 * NP + q] : 0.0;
            T4 v;
            v.x = ok ? (T)src[3 * NP + q] : T(0);
            v.y = ok ? (T)src[4 * NP + q] : T(0);
            v.z = ok ? (T)src[5 * NP + q] : T(0);
            v.w = ok ? (T)src[6 * NP + q] : T(0);
            s_v[idx] = v;
        }
        __syncthreads();

        const int ia = i0 + il, ib = i0 + il + HALF, j = j0 + jl;
        const bool live_a = ia < job.nr && j < job.nc;
        const bool live_b = ib < job.nr && j < job.nc;
        if (live_a) {
            T re_a = 0, im_a = 0, re_b = 0, im_b = 0;
            const double *pa = p_t + il * PS;
            const double *pb = p_t + (il + HALF) * PS;
            const T *va = v_t + il * VS;
            const T *vb = v_t + (il + HALF) * VS;
            const double2 *sxy = s_xy + jl * NP;
            const double *sz = s_z + jl * NP;
            const T4 *sv = s_v + jl * NP;
            if (r_near2 > 0.0) {
                bool near = false;
#pragma unroll
                for (int a = 0; a < 2; ++a)
#pragma unroll
                    for (int b = 0; b < 2; ++b) {
                        const double2 xy = sxy[b * Q];
                        const double z = sz[b * Q];
                        double dx = pa[a * Q] - xy.x, dy = pa[NP + a * Q] - xy.y, dz = pa[2 * NP + a * Q] - z;
                        near |= dx * dx + dy * dy + dz * dz < r_near2;
                        if (live_b) {
                            dx = pb[a * Q] - xy.x; dy = pb[NP + a * Q] - xy.y; dz = pb[2 * NP + a * Q] - z;
                            near |= dx * dx + dy * dy + dz * dz < r_near2;
                        }
                    }
                if (near) atomicOr(flags, 1);
            }
#pragma unroll 1
            for (int p = 0; p < NP; ++p) {
                const double xa = pa[p], ya = pa[NP + p], za = pa[2 * NP + p];
                const double xb = pb[p], yb = pb[NP + p], zb = pb[2 * NP + p];
                const T uxa = k * va[p], uya = k * va[NP + p], uza = k * va[2 * NP + p];
                const T da = kinv * va[3 * NP + p];
                const T uxb = k * vb[p], uyb = k * vb[NP + p], uzb = k * vb[2 * NP + p];
                const T db = kinv * vb[3 * NP + p];
#pragma unroll 2
                for (int q = 0; q < NP; ++q) {
                    const double2 xy = sxy[q];
                    const double z = sz[q];
                    const T4 v = sv[q];
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const double dx = (h ? xb : xa) - xy.x;
                        const double dy = (h ? yb : ya) - xy.y;
                        const double dz = (h ? zb : za) - z;
                        const double R2 = fma(dx, dx, fma(dy, dy, dz * dz));
                        T rinv, sn, cs;
                        int quad;
                        if constexpr (sizeof(T) == 8) {
                            rinv = rsqrt(R2);
                            const double g = split_quarter(R2 * rinv * kturn, &quad);
                            sincos_2pi(g, quad, &sn, &cs);
                        } else {
                            const float y = rsqrtf((float)R2);
                            const double yd = (double)y;
                            const double R0 = R2 * yd;
                            const double R = fma(fma(-R0, R0, R2), 0.5 * yd, R0);
                            const double g = split_quarter(R * kturn, &quad);
                            sincos_2pi((float)g, quad, &sn, &cs);
                            rinv = y;
                        }
                        const T ux = h ? uxb : uxa, uy = h ? uyb : uya, uz = h ? uzb : uza;
                        const T dd = h ? db : da;
                        const T A = fma(dd, v.w, -fma(ux, v.x, fma(uy, v.y, uz * v.z)));
                        const T t = A * rinv;
                        if (h) {
                            re_b = fma(t, sn, re_b);
                            im_b = fma(t, cs, im_b);
                        } else {
                            re_a = fma(t, sn, re_a);
                            im_a = fma(t, cs, im_a);
                        }
                    }
                }
            }
            C2 za_, zb_;
            za_.x = scale * re_a;
            za_.y = scale * im_a;
            zb_.x = scale * re_b;
            zb_.y = scale * im_b;
            C2 *out = reinterpret_cast<C2 *>(job.out);
            if (!job.trans) {
                out[ia + (size_t)j * job.ld] = za_;
                if (live_b) out[ib + (size_t)j * job.ld] = zb_;
            } else {
                out[j + (size_t)ia * job.ld] = za_;
                if (live_b) out[j + (size_t)ib * job.ld] = zb_;
            }
        }
        __syncthreads();
    }
}

template <typename T, int Q, int TM, int TN>
static int launch2_t(const double *rec, const FillParams &p, const FillJob *d_jobs,
                     const int *d_prefix, int njobs, int total_tiles, int *d_flags,
                     cudaStream_t stream) {
    constexpr int NP = 2 * Q;
    constexpr int PS = (3 * NP) | 1;
    constexpr int VS = (4 * NP) | 1;
    constexpr int NT = TM / 2 * TN;
    const size_t smem = (sizeof(double2) + sizeof(double) + 4 * sizeof(T)) * (size_t)TN * NP +
                        (sizeof(double) * PS + sizeof(T) * VS) * (size_t)TM + 16;
    auto kern = p.gates ? fill2_kernel<T, Q, TM, TN, true> : fill2_kernel<T, Q, TM, TN, false>;
    PSKEL_TRY(ensure_smem_attr(kern, smem));
    int per_sm = 0;
    PSKEL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem));
    if (per_sm < 1) per_sm = 1;
    long long grid = p.persistent ? (long long)sm_count() * per_sm : (long long)total_tiles;
    if (grid > total_tiles) grid = total_tiles;
    if (grid < 1) return PSKEL_OK;
    const double pi = 3.14159265358979323846;
    kern<<<(int)grid, NT, smem, stream>>>(rec, rec, d_jobs, d_prefix, njobs, total_tiles, (T)p.k,
                                          (T)(1.0 / p.k), p.k / (2.0 * pi), (T)(p.eta / (4.0 * pi)),
                                          p.r_near > 0 ? p.r_near * p.r_near : 0.0, d_flags, p.gates);
    PSKEL_LAUNCHED(1);
    return PSKEL_OK;
}

template <typename T, int Q, int TM, int TN, int SPLIT>
static int launch_t(const double *rec_t, const double *rec_s, const FillParams &p,
                    const FillJob *d_jobs, const int *d_prefix, int njobs, int total_tiles,
                    int *d_flags, cudaStream_t stream) {
    constexpr int NP = 2 * Q;
    constexpr int PS = (3 * NP) | 1;
    constexpr int VS = (4 * NP) | 1;
    constexpr int NT = TM * TN * SPLIT;
    const size_t smem = (sizeof(double) * PS + sizeof(T) * VS) * (size_t)(TM + TN) + 16;
    auto kern = p.gates ? fill_kernel<T, Q, TM, TN, SPLIT, true> : fill_kernel<T, Q, TM, TN, SPLIT, false>;
    PSKEL_TRY(ensure_smem_attr(kern, smem));
    int per_sm = 0;
    PSKEL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem));
    if (per_sm < 1) per_sm = 1;
    long long grid = p.persistent ? (long long)sm_count() * per_sm : (long long)total_tiles;
    if (grid > total_tiles) grid = total_tiles;
    if (grid < 1) return PSKEL_OK;
    const double pi = 3.14159265358979323846;
    const T k = (T)p.k;
    const T kinv = (T)(1.0 / p.k);
    const double kphase = sizeof(T) == 8 ? p.k / pi : p.k / (2.0 * pi);
    const T scale = (T)(p.eta / (4.0 * pi));
    const double rn2 = p.r_near > 0 ? p.r_near * p.r_near : 0.0;
    kern<<<(int)grid, NT, smem, stream>>>(rec_t, rec_s, d_jobs, d_prefix, njobs, total_tiles, k,
                                          kinv, kphase, scale, rn2, d_flags, p.gates);
    PSKEL_LAUNCHED(1);
    return PSKEL_OK;
}

int fill_tile_shape(int precision, int q, int split, int *tm, int *tn) {
    (void)q;
    if (split <= 0) {  // default kernel: 64 rows (two per thread) x 8 columns
        *tm = 64;
        *tn = 8;
        return PSKEL_OK;
    }
    if (precision == PSKEL_C128) {
        *tm = 16;
        *tn = split == 1 ? 16 : (split == 2 ? 8 : 4);
    } else {
        *tm = split == 1 ? 32 : 16;
        *tn = split == 1 ? 8 : (split == 2 ? 8 : 4);
    }
    return PSKEL_OK;
}

int launch_fill(const DevMesh &mesh, const FillParams &p, const FillJob *d_jobs,
                const int *d_tile_prefix, int njobs, int total_tiles, int *d_flags,
                cudaStream_t stream) {
    if (total_tiles <= 0 || njobs <= 0) return PSKEL_OK;
    if (p.q_test != p.q_src || (p.q_test != 1 && p.q_test != 7)) {
        set_error(PSKEL_ERR_ARG, "fill: q_test and q_src must both be 1 or both be 7");
        return PSKEL_ERR_ARG;
    }
    const DevMesh &m = mesh;
    const MeshRecords &rec = const_cast<DevMesh &>(m).records(p.q_test);
    if (rec.q != p.q_test) {
        set_error(PSKEL_ERR_STATE, "fill: records for Q=%d not built", p.q_test);
        return PSKEL_ERR_STATE;
    }
    const int split = p.split;
    const double *r64 = rec.f64.as<double>();
    if (split <= 0) {
        if (p.precision == PSKEL_C128) {
            if (p.q_test == 7)
                return launch2_t<double, 7, 64, 8>(r64, p, d_jobs, d_tile_prefix, njobs, total_tiles, d_flags, stream);
            return launch2_t<double, 1, 64, 8>(r64, p, d_jobs, d_tile_prefix, njobs, total_tiles, d_flags, stream);
        }
        if (p.q_test == 7)
            return launch2_t<float, 7, 64, 8>(r64, p, d_jobs, d_tile_prefix, njobs, total_tiles, d_flags, stream);
        return launch2_t<float, 1, 64, 8>(r64, p, d_jobs, d_tile_prefix, njobs, total_tiles, d_flags, stream);
    }
#define PSKEL_FILL_CASE(T, REC, Q, TM, TN, S)                                                   \
    return launch_t<T, Q, TM, TN, S>(REC, REC, p, d_jobs, d_tile_prefix, njobs, total_tiles,   \
                                     d_flags, stream)
    if (p.precision == PSKEL_C128) {
        if (p.q_test == 7) {
            if (split == 1) PSKEL_FILL_CASE(double, r64, 7, 16, 16, 1);
            if (split == 2) PSKEL_FILL_CASE(double, r64, 7, 16, 8, 2);
            PSKEL_FILL_CASE(double, r64, 7, 16, 4, 4);
        } else {
            if (split == 1) PSKEL_FILL_CASE(double, r64, 1, 16, 16, 1);
            if (split == 2) PSKEL_FILL_CASE(double, r64, 1, 16, 8, 2);
            PSKEL_FILL_CASE(double, r64, 1, 16, 4, 4);
        }
    } else {
        if (p.q_test == 7) {
            if (split == 1) PSKEL_FILL_CASE(float, r64, 7, 32, 8, 1);
            if (split == 2) PSKEL_FILL_CASE(float, r64, 7, 16, 8, 2);
            PSKEL_FILL_CASE(float, r64, 7, 16, 4, 4);
        } else {
            if (split == 1) PSKEL_FILL_CASE(float, r64, 1, 32, 8, 1);
            if (split == 2) PSKEL_FILL_CASE(float, r64, 1, 16, 8, 2);
            PSKEL_FILL_CASE(float, r64, 1, 16, 4, 4);
        }
    }
#undef PSKEL_FILL_CASE
}

// ============================================================ triangle-moment fill
// Z(group, cols) for a group of RWG functions with a known triangle list. For far interactions
// every point pair costs the same Green's function evaluation whichever RWG it is weighted for,
// and the RWG functions of a group share their triangles (about 2.5 RWG references per
// triangle on a closed surface). So G is evaluated once per (triangle t of the group, column
// RWG n) over the Q x 2Q point pairs and reduced to five moments, in coordinates local to the
// centroid c_t of t (x' = x - c_t) so that nothing cancels in FP32:
//     A0 = sum_p w_p S0_p,  Bx = sum_p w_p x'_p . S1_p,  Cv = sum_p w_p S1_p,
//     S0_p = sum_q G(x_p, y_q) e_q,  S1_p = sum_q G(x_p, y_q) v_q   (e, v: source record d, u)
// and each RWG m of the group that uses t as its side a (sign s_a, free vertex v_a, length l_m)
// receives   s_a l_m [ A0 / k - (k/2) (Bx - (v_a - c_t) . Cv) ],
// which is the per-entry sum sum_p sum_q G [d_p e_q / k - k u_p . v_q] regrouped. A CTA owns one
// job and kTriFillCols columns: it stages the column records, loops over (triangle, column)
// items, scatters the two to three contributions of each item into a shared-memory tile of the
// block (shared-memory atomics; each entry receives exactly two) and writes the tile once.
// Weights of the rule by point class: the centroid (point 0) and the two orbits of three
// points (1-3, 4-6) of the 7-point rule; Q = 1 uses w0 = 1.
struct TriWeights {
    double w0, w1, w2;
};

// OFS (complex-FP32 variant only): the point-pair geometry in FP32 offsets instead of FP64. Per
// item the vector D = c_t - y_0 from the source RWG's first point to the triangle centroid, |D|
// and the phase of |D| reduced to a fraction of a turn are FP64; per pair, with e = x'_p - (y_q - y_0)
// (both small), R^2 = |D|^2 + u with u = e . (2 D + e), and R - |D| = u / (R + |D|), all FP32:
// the phase keeps an absolute error of ~1e-7 turn without FP64 arithmetic in the pair loop.
template <typename T, int Q, int TN, bool OFS = false, bool GATED = false>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 3)
    tri_fill_kernel(const double *__restrict__ tri_rec, const double *__restrict__ rec_s,
                    const double *__restrict__ edges, const double *__restrict__ vertex,
                    const double *__restrict__ ln, const GroupFillJob *__restrict__ jobs,
                    const int *__restrict__ tile_prefix, int njobs, int total_tiles, T k,
                    T kinv, double kturn, T scale, TriWeights wq, const int *const *__restrict__ gates) {
    constexpr int NP = 2 * Q;
    constexpr int RS = (7 * NP) | 1;
    constexpr int TS = tri_stride(Q);
    using C2 = typename Cplx<T>::type;
    using T4 = typename Vec4<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *s_xy = reinterpret_cast<double2 *>(smem_raw);   // TN x NP
    double *s_z = reinterpret_cast<double *>(s_xy + TN * NP);  // TN x NP
    T4 *s_v = reinterpret_cast<T4 *>(s_z + TN * NP);           // TN x NP
    float4 *s_d = reinterpret_cast<float4 *>(s_v + TN * NP);   // TN x NP (OFS: y_q - y_0)
    T *zs = reinterpret_cast<T *>(s_d + (OFS ? TN * NP : 0));   // 2 x (largest m) x TN

    for (int tile = blockIdx.x; tile < total_tiles; tile += gridDim.x) {
        const int jb = find_job(tile_prefix, njobs, tile);
        if constexpr (GATED) {
            if (*gates[jb] == 0) continue;  // uniform over the CTA
        }
        const GroupFillJob job = jobs[jb];
        const int tcols = job.tc > 0 && job.tc < TN ? job.tc : TN;  // this job's tile width
        const int j0 = (tile - tile_prefix[jb]) * tcols;
        for (int idx = threadIdx.x; idx < tcols * NP; idx += blockDim.x) {
            const int c = idx / NP, q = idx - c * NP;
            const int col = j0 + c;
            const bool ok = col < job.nc;
            const double *src = rec_s + (size_t)(ok ? job.cols[col] : 0) * RS;
            s_xy[idx] = make_double2(ok ? src[q] : 0.0, ok ? src[NP + q] : 0.0);
            s_z[idx] = ok ? src[2 * NP + q] : 0.0;
            T4 v;
            v.x = ok ? (T)src[3 * NP + q] : T(0);
            v.y = ok ? (T)src[4 * NP + q] : T(0);
            v.z = ok ? (T)src[5 * NP + q] : T(0);
            v.w = ok ? (T)src[6 * NP + q] : T(0);
            s_v[idx] = v;
            if (OFS) {
                const float dx = ok ? (float)(src[q] - src[0]) : 0.f;
                const float dy = ok ? (float)(src[NP + q] - src[NP]) : 0.f;
                const float dz = ok ? (float)(src[2 * NP + q] - src[2 * NP]) : 0.f;
                s_d[idx] = make_float4(dx, dy, dz, fmaf(dx, dx, fmaf(dy, dy, dz * dz)));
            }
        }
        for (int idx = threadIdx.x; idx < 2 * job.m * tcols; idx += blockDim.x) zs[idx] = T(0);
        __syncthreads();

        const int items = job.nt * tcols;
        for (int it = threadIdx.x; it < items; it += blockDim.x) {
            const int t = it % job.nt, j = it / job.nt;
            if (j0 + j >= job.nc) continue;
            const double *tr = tri_rec + (size_t)job.tris[t] * TS;
            const double cx = tr[3 * Q], cy = tr[3 * Q + 1], cz = tr[3 * Q + 2];
            const double2 *sxy = s_xy + j * NP;
            const double *sz = s_z + j * NP;
            const T4 *sv = s_v + j * NP;
            T a0r = 0, a0i = 0, bxr = 0, bxi = 0;
            T cvr[3] = {0, 0, 0}, cvi[3] = {0, 0, 0};
            // OFS: item-level FP64 geometry from the source RWG's first point y_0
            float D2x = 0.f, D2y = 0.f, D2z = 0.f, DDf = 0.f, Dnf = 0.f, ph0 = 0.f;
            if constexpr (OFS) {
                const double Dx = cx - sxy[0].x, Dy = cy - sxy[0].y, Dz = cz - sz[0];
                const double DD = fma(Dx, Dx, fma(Dy, Dy, Dz * Dz));
                const double Dn = sqrt(DD);
                const double ph = Dn * kturn;
                D2x = (float)(2.0 * Dx);
                D2y = (float)(2.0 * Dy);
                D2z = (float)(2.0 * Dz);
                DDf = (float)DD;
                Dnf = (float)Dn;
                ph0 = (float)(ph - floor(ph));
            }
            const float kturnf = (float)kturn;
            const float4 *sd = s_d + j * NP;
#pragma unroll 1
            for (int p = 0; p < Q; ++p) {
                const double x = tr[3 * p], y = tr[3 * p + 1], z = tr[3 * p + 2];
                T s0r = 0, s0i = 0, s1r[3] = {0, 0, 0}, s1i[3] = {0, 0, 0};
                const float ex0 = (float)(x - cx), ey0 = (float)(y - cy), ez0 = (float)(z - cz);
                // OFS, per test point: A_p = D + x'_p and c_p = 2 D . x'_p + |x'_p|^2, so that per
                // pair u = |R|^2 - |D|^2 = c_p + |d_q|^2 - 2 A_p . d_q (d_q = y_q - y_0)
                const float Ax = fmaf(0.5f, D2x, ex0), Ay = fmaf(0.5f, D2y, ey0), Az = fmaf(0.5f, D2z, ez0);
                const float cp = fmaf(ex0, fmaf(1.0f, D2x, ex0), fmaf(ey0, D2y + ey0, ez0 * (D2z + ez0)));
#pragma unroll(OFS ? 7 : 2)
                for (int q = 0; q < NP; ++q) {
                    T rinv, sn, cs;
                    int quad;
                    if constexpr (OFS) {
                        const float4 d = sd[q];  // (d_q, |d_q|^2)
                        const float dot = fmaf(Ax, d.x, fmaf(Ay, d.y, Az * d.z));
                        const float u = fmaf(-2.0f, dot, cp + d.w);
                        const float R2f = DDf + u;
                        const float ri = rsqrtf(R2f);
                        const float corr = __fdividef(u, fmaf(R2f, ri, Dnf));  // R - |D|
                        const float turns = fmaf(corr, kturnf, ph0);
                        // half-turn reduction: turns = n/2 + g, |g| <= 1/4; sin and cos take (-1)^n,
                        // folded into the sign of 1/R
                        const float tm = fmaf(turns, 2.0f, 12582912.0f);     // 1.5 * 2^23
                        const float g = fmaf(tm - 12582912.0f, -0.5f, turns);
                        sincos_2pi_half(g, &sn, &cs);
                        rinv = __int_as_float(__float_as_int(ri) ^ (__float_as_int(tm) << 31));
                        (void)quad;
                    } else {
                    const double2 xy = sxy[q];
                    const double dx = x - xy.x, dy = y - xy.y, dz = z - sz[q];
                    const double R2 = fma(dx, dx, fma(dy, dy, dz * dz));
                    if constexpr (sizeof(T) == 8) {
                        rinv = rsqrt(R2);
                        const double g = split_quarter(R2 * rinv * kturn, &quad);
                        sincos_2pi(g, quad, &sn, &cs);
                    } else {
                        const float yy = rsqrtf((float)R2);
                        const double yd = (double)yy;
                        const double R0 = R2 * yd;
                        const double R = fma(fma(-R0, R0, R2), 0.5 * yd, R0);
                        const double g = split_quarter(R * kturn, &quad);
                        sincos_2pi((float)g, quad, &sn, &cs);
                        rinv = yy;
                    }
                    }
                    const T gr = rinv * sn, gi = rinv * cs;  // G = (sin kR + j cos kR) / R
                    const T4 v = sv[q];
                    s0r = fma(gr, v.w, s0r);
                    s0i = fma(gi, v.w, s0i);
                    s1r[0] = fma(gr, v.x, s1r[0]);
                    s1i[0] = fma(gi, v.x, s1i[0]);
                    s1r[1] = fma(gr, v.y, s1r[1]);
                    s1i[1] = fma(gi, v.y, s1i[1]);
                    s1r[2] = fma(gr, v.z, s1r[2]);
                    s1i[2] = fma(gi, v.z, s1i[2]);
                }
                const T w = (T)(p == 0 ? wq.w0 : (p < 4 ? wq.w1 : wq.w2));
                const T xl[3] = {(T)(x - cx), (T)(y - cy), (T)(z - cz)};
                a0r = fma(w, s0r, a0r);
                a0i = fma(w, s0i, a0i);
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    cvr[d] = fma(w, s1r[d], cvr[d]);
                    cvi[d] = fma(w, s1i[d], cvi[d]);
                    bxr = fma(w * xl[d], s1r[d], bxr);
                    bxi = fma(w * xl[d], s1i[d], bxi);
                }
            }
            const int *ad = job.adj + 3 * t;
#pragma unroll
            for (int u = 0; u < 3; ++u) {
                const int a = ad[u];
                if (a < 0) continue;
                const int ml = a >> 1, side = a & 1;
                T vl[3], sl;
                if (job.use) {  // free vertex - centroid and s l, looked up once per group
                    const double *uz = job.use + 4 * (3 * (size_t)t + u);
                    vl[0] = (T)uz[0];
                    vl[1] = (T)uz[1];
                    vl[2] = (T)uz[2];
                    sl = (T)uz[3];
                } else {
                    const int e = job.rows[ml];
                    const int vo = (int)edges[4 * (size_t)e + 2 + side] - 1;
                    vl[0] = (T)(vertex[3 * (size_t)vo] - cx);
                    vl[1] = (T)(vertex[3 * (size_t)vo + 1] - cy);
                    vl[2] = (T)(vertex[3 * (size_t)vo + 2] - cz);
                    sl = (side ? -1 : 1) * (T)ln[e];
                }
                const T hk = (T)0.5 * k;
                T br = bxr, bi = bxi;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    br = fma(-vl[d], cvr[d], br);
                    bi = fma(-vl[d], cvi[d], bi);
                }
                const T vr = sl * fma(a0r, kinv, -hk * br);
                const T vi = sl * fma(a0i, kinv, -hk * bi);
                atomicAdd(&zs[2 * (ml + j * job.m)], vr);
                atomicAdd(&zs[2 * (ml + j * job.m) + 1], vi);
            }
        }
        __syncthreads();
        C2 *out = reinterpret_cast<C2 *>(job.out);
        for (int idx = threadIdx.x; idx < job.m * tcols; idx += blockDim.x) {
            const int i = idx % job.m, j = idx / job.m;
            if (j0 + j >= job.nc) continue;
            C2 z;
            z.x = scale * zs[2 * idx];
            z.y = scale * zs[2 * idx + 1];
            if (!job.trans) out[i + (size_t)(j0 + j) * job.ld] = z;
            else out[(j0 + j) + (size_t)i * job.ld] = z;
        }
        __syncthreads();
    }
}

template <typename T, int Q, int TN, bool OFS = false>
static int launch_tri_t(const DevMesh &mesh, const MeshRecords &rec, const FillParams &p,
                        const GroupFillJob *d_jobs, const int *d_prefix, int njobs,
                        int total_tiles, cudaStream_t stream) {
    constexpr int NP = 2 * Q;
    const size_t rec_bytes =
        (sizeof(double2) + sizeof(double) + 4 * sizeof(T) + (OFS ? sizeof(float4) : 0)) * (size_t)TN * NP;
    const int rows = p.max_rows > 0 && p.max_rows < kTriFillMaxRows ? p.max_rows : kTriFillMaxRows;
    const size_t smem = rec_bytes + 2 * sizeof(T) * (size_t)rows * TN + 16;
    auto kern = p.gates ? tri_fill_kernel<T, Q, TN, OFS, true> : tri_fill_kernel<T, Q, TN, OFS, false>;
    PSKEL_TRY(ensure_smem_attr(kern, rec_bytes + 2 * sizeof(T) * (size_t)kTriFillMaxRows * TN + 16));
    int per_sm = 0;
    PSKEL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, smem));
    if (per_sm < 1) per_sm = 1;
    long long grid = p.persistent ? (long long)sm_count() * per_sm : (long long)total_tiles;
    if (grid > total_tiles) grid = total_tiles;
    if (grid < 1) return PSKEL_OK;
    double wall[7];
    quadrature_weights(Q, wall);
    TriWeights w{wall[0], Q == 7 ? wall[1] : 0.0, Q == 7 ? wall[4] : 0.0};
    const double pi = 3.14159265358979323846;
    kern<<<(int)grid, 256, smem, stream>>>(
        rec.tri.as<double>(), rec.f64.as<double>(), mesh.edges.as<double>(),
        mesh.vertex.as<double>(), mesh.ln.as<double>(), d_jobs, d_prefix, njobs, total_tiles,
        (T)p.k, (T)(1.0 / p.k), p.k / (2.0 * pi), (T)(p.eta / (4.0 * pi)), w, p.gates);
    PSKEL_LAUNCHED(1);
    return PSKEL_OK;
}

int launch_tri_fill(const DevMesh &mesh, const FillParams &p, const GroupFillJob *d_jobs,
                    const int *d_tile_prefix, int njobs, int total_tiles, cudaStream_t stream) {
    if (total_tiles <= 0 || njobs <= 0) return PSKEL_OK;
    if (p.q_test != p.q_src || (p.q_test != 1 && p.q_test != 7)) {
        set_error(PSKEL_ERR_ARG, "tri fill: q_test and q_src must both be 1 or both be 7");
        return PSKEL_ERR_ARG;
    }
    const MeshRecords &rec = const_cast<DevMesh &>(mesh).records(p.q_test);
    if (rec.q != p.q_test) {
        set_error(PSKEL_ERR_STATE, "tri fill: records for Q=%d not built", p.q_test);
        return PSKEL_ERR_STATE;
    }
#define PSKEL_TRI(T, Q, TN) \
    return launch_tri_t<T, Q, TN>(mesh, rec, p, d_jobs, d_tile_prefix, njobs, total_tiles, stream)
#define PSKEL_TRI_OFS(Q, TN) \
    return launch_tri_t<float, Q, TN, true>(mesh, rec, p, d_jobs, d_tile_prefix, njobs, total_tiles, stream)
#define PSKEL_TRI_TN(T, Q)                     \
    do {                                       \
        if (p.tri_cols == 4) PSKEL_TRI(T, Q, 4);   \
        if (p.tri_cols == 16 || p.tri_cols == 0) PSKEL_TRI(T, Q, 16); \
        PSKEL_TRI(T, Q, 8);                    \
    } while (0)
    if (p.tri_cols != 0 && p.tri_cols != 4 && p.tri_cols != 8 && p.tri_cols != 16) {
        set_error(PSKEL_ERR_ARG, "tri fill: %d columns per tile (0 = balanced per job, 4, 8 or 16)", p.tri_cols);
        return PSKEL_ERR_ARG;
    }
    if (p.precision == PSKEL_C128) {
        if (p.q_test == 7) PSKEL_TRI_TN(double, 7);
        PSKEL_TRI_TN(double, 1);
    }
    if (p.geom32) {  // complex-FP32 fill with FP32 pair geometry
        if (p.q_test == 7) {
            if (p.tri_cols == 4) PSKEL_TRI_OFS(7, 4);
            if (p.tri_cols == 16 || p.tri_cols == 0) PSKEL_TRI_OFS(7, 16);
            PSKEL_TRI_OFS(7, 8);
        }
        if (p.tri_cols == 4) PSKEL_TRI_OFS(1, 4);
        if (p.tri_cols == 16 || p.tri_cols == 0) PSKEL_TRI_OFS(1, 16);
        PSKEL_TRI_OFS(1, 8);
    }
    if (p.q_test == 7) PSKEL_TRI_TN(float, 7);
    PSKEL_TRI_TN(float, 1);
#undef PSKEL_TRI_TN
#undef PSKEL_TRI_OFS
#undef PSKEL_TRI
}

// ---------------------------------------------------------------- diagnostics
// The fill's sin/cos of 2 pi t next to CUDA's sincospi(2 t), for tests of the polynomials: the
// quarter-turn forms in FP64 and FP32, CUDA's values, then the half-turn FP32 form of the
// complex-FP32 fill with FP32 pair geometry (t = n/2 + g, sign (-1)^n).
__global__ void diag_sincos_kernel(const double *t, int n, double *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int q;
    const double g = split_quarter(t[i], &q);
    double s, c;
    sincos_2pi(g, q, &s, &c);
    float sf, cf;
    sincos_2pi((float)g, q, &sf, &cf);
    double rs, rc;
    sincospi(2.0 * t[i], &rs, &rc);
    const double nh = rint(2.0 * t[i]);
    float sh, ch;
    sincos_2pi_half((float)(t[i] - 0.5 * nh), &sh, &ch);
    const float sg = ((long long)nh & 1) ? -1.0f : 1.0f;
    out[8 * i + 0] = s;
    out[8 * i + 1] = c;
    out[8 * i + 2] = sf;
    out[8 * i + 3] = cf;
    out[8 * i + 4] = rs;
    out[8 * i + 5] = rc;
    out[8 * i + 6] = sg * sh;
    out[8 * i + 7] = sg * ch;
}

}  // namespace pskel

extern "C" int pskel_diag_sincos(const double *t_dev, int n, double *out_dev) {
    using namespace pskel;
    if (!t_dev || !out_dev || n < 0) {
        set_error(PSKEL_ERR_ARG, "diag_sincos: bad arguments");
        return PSKEL_ERR_ARG;
    }
    if (n == 0) return PSKEL_OK;
    diag_sincos_kernel<<<(n + 255) / 256, 256>>>(t_dev, n, out_dev);
    PSKEL_LAUNCHED(1);
    return PSKEL_OK;
}
