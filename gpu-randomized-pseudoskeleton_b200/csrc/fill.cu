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
template <typename T, int Q, int TM, int TN, int SPLIT>
__global__ void __launch_bounds__(TM *TN *SPLIT, FillOcc<T>::value)
    fill_kernel(const double *__restrict__ rec_t, const double *__restrict__ rec_s,
                const FillJob *__restrict__ jobs, const int *__restrict__ tile_prefix, int njobs,
                int total_tiles, T k, T kinv, double kphase, T scale, double r_near2, int *flags) {
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
            reinterpret_cast<C2 *>(job.out)[i + (size_t)j * job.ld] = z;
        }
        __syncthreads();
    }
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
    auto kern = fill_kernel<T, Q, TM, TN, SPLIT>;
    static bool attr_set = false;
    if (!attr_set) {
        PSKEL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem));
        attr_set = true;
    }
    int per_sm = 0;
    PSKEL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem));
    if (per_sm < 1) per_sm = 1;
    long long grid = (long long)sm_count() * per_sm;
    if (grid > total_tiles) grid = total_tiles;
    if (grid < 1) return PSKEL_OK;
    const double pi = 3.14159265358979323846;
    const T k = (T)p.k;
    const T kinv = (T)(1.0 / p.k);
    const double kphase = sizeof(T) == 8 ? p.k / pi : p.k / (2.0 * pi);
    const T scale = (T)(p.eta / (4.0 * pi));
    const double rn2 = p.r_near > 0 ? p.r_near * p.r_near : 0.0;
    kern<<<(int)grid, NT, smem, stream>>>(rec_t, rec_s, d_jobs, d_prefix, njobs, total_tiles, k,
                                          kinv, kphase, scale, rn2, d_flags);
    PSKEL_LAUNCHED(1);
    return PSKEL_OK;
}

int fill_tile_shape(int precision, int q, int split, int *tm, int *tn) {
    (void)q;
    if (split <= 0) split = 1;
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
    const int split = p.split <= 0 ? 1 : p.split;
    const double *r64 = rec.f64.as<double>();
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

}  // namespace pskel
