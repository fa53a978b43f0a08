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
// Design (B200): the kernel is bound by the FP64 (c128) or FP32/MUFU (c64) pipes, not by
// memory. A CTA owns a TM x TN tile of one job; the TM test and TN source records are gathered
// once into shared memory (coalesced, odd record stride for conflict-free bank access), each
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

template <typename T>
__device__ __forceinline__ void green_sincos(T R, T kphase, T *s, T *c);

// FP64: sincospi(R k / pi) - the reduction by pi is exact, cheaper than sincos(kR).
template <>
__device__ __forceinline__ void green_sincos<double>(double R, double kpi, double *s, double *c) {
    sincospi(R * kpi, s, c);
}
// FP32: phase in turns t = R k / (2 pi); f = t - rint(t) in [-1/2, 1/2] is exact for the
// electrical sizes used here, so the fast hardware sin/cos sees |angle| <= pi.
template <>
__device__ __forceinline__ void green_sincos<float>(float R, float kturn, float *s, float *c) {
    const float t = R * kturn;
    const float f = t - rintf(t);
    __sincosf(f * 6.28318530717958647692f, s, c);
}

template <typename T> __device__ __forceinline__ T rsqrt_t(T x);
template <> __device__ __forceinline__ double rsqrt_t<double>(double x) { return rsqrt(x); }
template <> __device__ __forceinline__ float rsqrt_t<float>(float x) { return rsqrtf(x); }

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

template <typename T, int Q, int TM, int TN, int SPLIT>
__global__ void __launch_bounds__(TM *TN *SPLIT, FillOcc<T>::value)
    fill_kernel(const T *__restrict__ rec_t, const T *__restrict__ rec_s,
                const FillJob *__restrict__ jobs, const int *__restrict__ tile_prefix, int njobs,
                int total_tiles, T k, T kinv, T kphase, T scale, T r_near2, int *flags) {
    constexpr int NP = 2 * Q;
    constexpr int RS = (7 * NP) | 1;
    constexpr int NT = TM * TN * SPLIT;
    using C2 = typename Cplx<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *s_t = reinterpret_cast<T *>(smem_raw);  // TM records
    T *s_s = s_t + TM * RS;                    // TN records

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

        for (int idx = tid; idx < TM * RS; idx += NT) {
            const int r = idx / RS, f = idx - (idx / RS) * RS;
            const int row = i0 + r;
            s_t[idx] = row < job.nr ? rec_t[(size_t)job.rows[row] * RS + f] : T(0);
        }
        for (int idx = tid; idx < TN * RS; idx += NT) {
            const int r = idx / RS, f = idx - (idx / RS) * RS;
            const int col = j0 + r;
            s_s[idx] = col < job.nc ? rec_s[(size_t)job.cols[col] * RS + f] : T(0);
        }
        __syncthreads();

        const int i = i0 + il, j = j0 + jl;
        const bool live = i < job.nr && j < job.nc;
        T re = 0, im = 0;
        if (live) {
            const T *tr = s_t + il * RS;
            const T *sr = s_s + jl * RS;
            if (r_near2 > T(0) && ls == 0) {
                // point 0 of each side is the triangle centroid (Q = 1 and Q = 7 rules)
                bool near = false;
#pragma unroll
                for (int a = 0; a < 2; ++a)
#pragma unroll
                    for (int b = 0; b < 2; ++b) {
                        const T dx = tr[a * Q] - sr[b * Q];
                        const T dy = tr[NP + a * Q] - sr[NP + b * Q];
                        const T dz = tr[2 * NP + a * Q] - sr[2 * NP + b * Q];
                        near |= dx * dx + dy * dy + dz * dz < r_near2;
                    }
                if (near) atomicOr(flags, 1);
            }
#pragma unroll 1
            for (int p = 0; p < NP; ++p) {
                const T xp = tr[p], yp = tr[NP + p], zp = tr[2 * NP + p];
                const T ux = k * tr[3 * NP + p], uy = k * tr[4 * NP + p], uz = k * tr[5 * NP + p];
                const T dp = kinv * tr[6 * NP + p];
#pragma unroll 2
                for (int q = ls; q < NP; q += SPLIT) {
                    const T dx = xp - sr[q], dy = yp - sr[NP + q], dz = zp - sr[2 * NP + q];
                    const T R2 = fma(dx, dx, fma(dy, dy, dz * dz));
                    const T rinv = rsqrt_t<T>(R2);
                    const T R = R2 * rinv;
                    T sn, cs;
                    green_sincos<T>(R, kphase, &sn, &cs);
                    const T A = fma(dp, sr[6 * NP + q],
                                    -fma(ux, sr[3 * NP + q], fma(uy, sr[4 * NP + q], uz * sr[5 * NP + q])));
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
static int launch_t(const T *rec_t, const T *rec_s, const FillParams &p, const FillJob *d_jobs,
                    const int *d_prefix, int njobs, int total_tiles, int *d_flags,
                    cudaStream_t stream) {
    constexpr int NP = 2 * Q;
    constexpr int RS = (7 * NP) | 1;
    constexpr int NT = TM * TN * SPLIT;
    const size_t smem = sizeof(T) * (size_t)(TM + TN) * RS;
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
    const T kphase = (T)(sizeof(T) == 8 ? p.k / pi : p.k / (2.0 * pi));
    const T scale = (T)(p.eta / (4.0 * pi));
    const T rn2 = (T)(p.r_near > 0 ? p.r_near * p.r_near : 0.0);
    kern<<<(int)grid, NT, smem, stream>>>(rec_t, rec_s, d_jobs, d_prefix, njobs, total_tiles, k,
                                          kinv, kphase, scale, rn2, d_flags);
    PSKEL_CUDA(cudaGetLastError());
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
    const float *r32 = rec.f32.as<float>();
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
            if (split == 1) PSKEL_FILL_CASE(float, r32, 7, 32, 8, 1);
            if (split == 2) PSKEL_FILL_CASE(float, r32, 7, 16, 8, 2);
            PSKEL_FILL_CASE(float, r32, 7, 16, 4, 4);
        } else {
            if (split == 1) PSKEL_FILL_CASE(float, r32, 1, 32, 8, 1);
            if (split == 2) PSKEL_FILL_CASE(float, r32, 1, 16, 8, 2);
            PSKEL_FILL_CASE(float, r32, 1, 16, 4, 4);
        }
    }
#undef PSKEL_FILL_CASE
}

}  // namespace pskel
