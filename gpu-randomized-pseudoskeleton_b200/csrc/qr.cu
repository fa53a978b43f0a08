// Batched Householder QR of tall complex FP64 matrices and the application of Q to small
// blocks: the two QR factorisations of the recompression (codes/ACA_vs_CUR/seed/svd_compress.m:
// 19-23, qr(C) and qr(R^H), there through the unshipped qr_cbd).
//
// QR: one CTA per matrix, in shared memory when it fits (else in place in global memory). Step k
// builds the reflector H_k = I - coef_k v_k v_k^H with v_k = x - beta e_1 from column k (one
// warp: norm and beta = -e^{i arg x_0} |x|), then a lane team per remaining column applies it
// (dot product with a shuffle reduction, then the update). The tail of v_k stays below the
// diagonal of A, v_k(0) and coef_k go to side arrays, R (n x n, zero below the diagonal) is
// written out separately.
//
// Apply: Y(:, j) = Q [Z(:, j); 0] = H_0 H_1 ... H_{n-1} [Z(:, j); 0], one lane team per column,
// the column held in the team's registers when m <= 256 (else updated in place in Y).
#include <algorithm>

#include "pskel_internal.cuh"

namespace pskel {

static constexpr size_t kQrSmem = 200 * 1024;
static constexpr int kQrThreads = 512;
static constexpr int kApplyRows = 8;  // rows per lane in the register path (team of 32: m <= 256)

__device__ __forceinline__ int qr_team(int m) {
    int t = 1;
    while (t < 32 && 2 * t * 2 <= m) t <<= 1;  // about two rows per lane at least
    return t;
}

template <bool SMEM>
__global__ void __launch_bounds__(kQrThreads) qr_kernel(const QrJob *__restrict__ jobs) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const QrJob job = jobs[blockIdx.x];
    const int m = job.m, n = job.n;
    double2 *A = SMEM ? reinterpret_cast<double2 *>(smem_raw) : job.A;
    __shared__ double s_coef;
    __shared__ double2 s_v0;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (SMEM) {
        for (int i = tid; i < m * n; i += blockDim.x) A[i] = job.A[i];
        __syncthreads();
    }
    const int team = qr_team(m);
    const int teams = blockDim.x / team;
    const int tt = tid / team, tg = tid % team;
    for (int k = 0; k < n; ++k) {
        if (warp == 0) {
            double x2 = 0;
            for (int i = k + lane; i < m; i += 32) {
                const double2 a = A[i + (size_t)k * m];
                x2 = fma(a.x, a.x, fma(a.y, a.y, x2));
            }
            for (int o = 16; o > 0; o >>= 1) x2 += __shfl_xor_sync(0xffffffffu, x2, o);
            if (lane == 0) {
                const double2 x0 = A[k + (size_t)k * m];
                const double ax0 = hypot(x0.x, x0.y);
                const double xn = sqrt(x2);
                double2 beta = make_double2(0.0, 0.0), v0 = make_double2(0.0, 0.0);
                double coef = 0.0;
                if (xn > 0.0) {
                    const double2 ph = ax0 > 0 ? make_double2(x0.x / ax0, x0.y / ax0) : make_double2(1.0, 0.0);
                    beta = make_double2(-ph.x * xn, -ph.y * xn);
                    v0 = make_double2(x0.x - beta.x, x0.y - beta.y);
                    const double v2 = x2 - ax0 * ax0 + (v0.x * v0.x + v0.y * v0.y);
                    coef = v2 > 0 ? 2.0 / v2 : 0.0;
                }
                job.v0[k] = v0;
                job.coef[k] = coef;
                s_v0 = v0;
                s_coef = coef;
                A[k + (size_t)k * m] = beta;  // R(k, k)
            }
        }
        __syncthreads();
        const double coef = s_coef;
        const double2 v0 = s_v0;
        const double2 *v = A + (size_t)k * m;
        if (coef != 0.0) {
            for (int j0 = k + 1; j0 < n; j0 += teams) {
                const int j = j0 + tt;
                double2 *a = A + (size_t)j * m;
                double dr = 0, di = 0;
                if (j < n)
                    for (int i = k + tg; i < m; i += team) {  // v^H a_j
                        const double2 x = i == k ? v0 : v[i], y = a[i];
                        dr = fma(x.x, y.x, fma(x.y, y.y, dr));
                        di = fma(x.x, y.y, fma(-x.y, y.x, di));
                    }
                for (int o = 1; o < team; o <<= 1) {
                    dr += __shfl_xor_sync(0xffffffffu, dr, o);
                    di += __shfl_xor_sync(0xffffffffu, di, o);
                }
                if (j < n) {
                    const double fr = coef * dr, fi = coef * di;
                    for (int i = k + tg; i < m; i += team) {
                        const double2 x = i == k ? v0 : v[i];
                        double2 y = a[i];
                        y.x -= fr * x.x - fi * x.y;
                        y.y -= fr * x.y + fi * x.x;
                        a[i] = y;
                    }
                }
            }
        }
        __syncthreads();
    }
    // R out (zero below the diagonal); the reflector tails back to global memory
    for (int idx = tid; idx < n * n; idx += blockDim.x) {
        const int i = idx % n, j = idx / n;
        job.R[idx] = i <= j ? A[i + (size_t)j * m] : make_double2(0.0, 0.0);
    }
    if (SMEM)
        for (int i = tid; i < m * n; i += blockDim.x) job.A[i] = A[i];
}

template <bool REG>
__global__ void __launch_bounds__(256) apply_q_kernel(const ApplyQJob *__restrict__ jobs) {
    const ApplyQJob job = jobs[blockIdx.x];
    const int m = job.m, n = job.n;
    const int kcols = job.kp ? min(*job.kp, job.k) : job.k;
    const int team = REG ? 32 : qr_team(m);
    const int teams = blockDim.x / team;
    const int tt = threadIdx.x / team, tg = threadIdx.x % team;
    for (int j0 = 0; j0 < kcols; j0 += teams) {
        const int j = j0 + tt;
        const bool on = j < kcols;
        if (REG) {
            double2 y[kApplyRows];
#pragma unroll
            for (int e = 0; e < kApplyRows; ++e) {
                const int i = tg + e * team;
                y[e] = (on && i < n) ? job.Z[i + (size_t)j * job.ldz] : make_double2(0.0, 0.0);
            }
            for (int k = n - 1; k >= 0; --k) {
                const double coef = job.coef[k];
                const double2 v0 = job.v0[k];
                double dr = 0, di = 0;
#pragma unroll
                for (int e = 0; e < kApplyRows; ++e) {
                    const int i = tg + e * team;
                    if (i >= k && i < m) {
                        const double2 x = i == k ? v0 : job.A[i + (size_t)k * m];
                        dr = fma(x.x, y[e].x, fma(x.y, y[e].y, dr));
                        di = fma(x.x, y[e].y, fma(-x.y, y[e].x, di));
                    }
                }
                for (int o = 1; o < team; o <<= 1) {
                    dr += __shfl_xor_sync(0xffffffffu, dr, o);
                    di += __shfl_xor_sync(0xffffffffu, di, o);
                }
                const double fr = coef * dr, fi = coef * di;
#pragma unroll
                for (int e = 0; e < kApplyRows; ++e) {
                    const int i = tg + e * team;
                    if (i >= k && i < m) {
                        const double2 x = i == k ? v0 : job.A[i + (size_t)k * m];
                        y[e].x -= fr * x.x - fi * x.y;
                        y[e].y -= fr * x.y + fi * x.x;
                    }
                }
            }
            if (on) {
#pragma unroll
                for (int e = 0; e < kApplyRows; ++e) {
                    const int i = tg + e * team;
                    if (i < m) job.Y[i + (size_t)j * job.ldy] = y[e];
                }
            }
        } else {
            double2 *y = job.Y + (size_t)(on ? j : 0) * job.ldy;
            if (on)
                for (int i = tg; i < m; i += team) y[i] = i < n ? job.Z[i + (size_t)j * job.ldz] : make_double2(0.0, 0.0);
            for (int k = n - 1; k >= 0; --k) {
                const double coef = job.coef[k];
                const double2 v0 = job.v0[k];
                double dr = 0, di = 0;
                if (on)
                    for (int i = k + tg; i < m; i += team) {
                        const double2 x = i == k ? v0 : job.A[i + (size_t)k * m];
                        const double2 yy = y[i];
                        dr = fma(x.x, yy.x, fma(x.y, yy.y, dr));
                        di = fma(x.x, yy.y, fma(-x.y, yy.x, di));
                    }
                for (int o = 1; o < team; o <<= 1) {
                    dr += __shfl_xor_sync(0xffffffffu, dr, o);
                    di += __shfl_xor_sync(0xffffffffu, di, o);
                }
                if (on) {
                    const double fr = coef * dr, fi = coef * di;
                    for (int i = k + tg; i < m; i += team) {
                        const double2 x = i == k ? v0 : job.A[i + (size_t)k * m];
                        double2 yy = y[i];
                        yy.x -= fr * x.x - fi * x.y;
                        yy.y -= fr * x.y + fi * x.x;
                        y[i] = yy;
                    }
                }
            }
        }
    }
}

static bool qr_fits(int m, int n) { return (size_t)m * n * sizeof(double2) <= kQrSmem; }

int batched_qr(const std::vector<QrJob> &h_jobs, cudaStream_t stream, DevBuf &scratch) {
    if (h_jobs.empty()) return PSKEL_OK;
    PSKEL_TRY(ensure_smem_attr(qr_kernel<true>, kQrSmem));
    // two launches: the jobs that fit in shared memory (grouped by size for the allocation) and
    // the rest in global memory
    std::vector<QrJob> fit, big;
    size_t smem = 0;
    int maxm = 1, maxn = 1;
    for (const QrJob &j : h_jobs) {
        if (qr_fits(j.m, j.n)) {
            fit.push_back(j);
            smem = std::max(smem, (size_t)j.m * j.n * sizeof(double2));
            maxm = std::max(maxm, j.m);
            maxn = std::max(maxn, j.n);
        } else {
            big.push_back(j);
        }
    }
    const size_t bytes = sizeof(QrJob) * (fit.size() + big.size());
    PSKEL_TRY(scratch.reserve(bytes + 256));
    QrJob *d = scratch.as<QrJob>();
    if (!fit.empty())
        PSKEL_CUDA(cudaMemcpyAsync(d, fit.data(), sizeof(QrJob) * fit.size(), cudaMemcpyHostToDevice, stream));
    if (!big.empty())
        PSKEL_CUDA(cudaMemcpyAsync(d + fit.size(), big.data(), sizeof(QrJob) * big.size(),
                                   cudaMemcpyHostToDevice, stream));
    auto threads_for = [](int m, int n) {
        int t = 1;
        while (t < 32 && 4 * t <= m) t <<= 1;
        int want = t * std::max(1, n - 1);
        want = (want + 31) / 32 * 32;
        return std::max(64, std::min(kQrThreads, want));
    };
    if (!fit.empty()) {
        qr_kernel<true><<<(unsigned)fit.size(), threads_for(maxm, maxn), smem, stream>>>(d);
        PSKEL_LAUNCHED(1);
    }
    if (!big.empty()) {
        int bm = 1, bn = 1;
        for (const QrJob &j : big) { bm = std::max(bm, j.m); bn = std::max(bn, j.n); }
        qr_kernel<false><<<(unsigned)big.size(), threads_for(bm, bn), 0, stream>>>(d + fit.size());
        PSKEL_LAUNCHED(1);
    }
    return PSKEL_OK;
}

int batched_apply_q(const std::vector<ApplyQJob> &h_jobs, cudaStream_t stream, DevBuf &scratch) {
    if (h_jobs.empty()) return PSKEL_OK;
    std::vector<ApplyQJob> reg, glob;
    for (const ApplyQJob &j : h_jobs) (j.m <= 32 * kApplyRows ? reg : glob).push_back(j);
    PSKEL_TRY(scratch.reserve(sizeof(ApplyQJob) * h_jobs.size() + 256));
    ApplyQJob *d = scratch.as<ApplyQJob>();
    if (!reg.empty())
        PSKEL_CUDA(cudaMemcpyAsync(d, reg.data(), sizeof(ApplyQJob) * reg.size(), cudaMemcpyHostToDevice, stream));
    if (!glob.empty())
        PSKEL_CUDA(cudaMemcpyAsync(d + reg.size(), glob.data(), sizeof(ApplyQJob) * glob.size(),
                                   cudaMemcpyHostToDevice, stream));
    if (!reg.empty()) {
        apply_q_kernel<true><<<(unsigned)reg.size(), 256, 0, stream>>>(d);
        PSKEL_LAUNCHED(1);
    }
    if (!glob.empty()) {
        apply_q_kernel<false><<<(unsigned)glob.size(), 256, 0, stream>>>(d + reg.size());
        PSKEL_LAUNCHED(1);
    }
    return PSKEL_OK;
}

}  // namespace pskel
