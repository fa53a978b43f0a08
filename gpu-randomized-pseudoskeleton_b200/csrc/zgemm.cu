// Batched complex FP64 GEMM for the small dense products of the CUR path
// (compressed matvec C (U (R x)), extra-row estimate, FP64 parts of the recompression).
// Replaces the reference's cublasZgemm calls (user_impedance_for_julia_cuda.cu:1929-1960).
//
// C_b = alpha op(A_b) op(B_b) + beta C_b for a list of jobs of different shapes; one CTA per
// 32 x 32 output tile, 256 threads x 4 outputs, K staged through shared memory in chunks of 16.
// The tile list of all jobs is flattened with a prefix array (like the fill).
#include "pskel_internal.cuh"
#include "zgemm.cuh"

namespace pskel {

__device__ __forceinline__ double2 load_op(const double2 *M, int ld, int op, int i, int k) {
    // element (i, k) of op(M)
    if (op == ZOP_N) return M[i + (size_t)k * ld];
    const double2 v = M[k + (size_t)i * ld];
    return op == ZOP_C ? make_double2(v.x, -v.y) : v;
}

__global__ void __launch_bounds__(256) zgemm_kernel(const ZgemmJob *__restrict__ jobs,
                                                    const int *__restrict__ prefix, int njobs) {
    int lo = 0, hi = njobs;
    const int tile = blockIdx.x;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (prefix[mid] <= tile) lo = mid; else hi = mid;
    }
    const ZgemmJob job = jobs[lo];
    const int local = tile - prefix[lo];
    const int tiles_m = (job.m + 31) / 32;
    const int i0 = (local % tiles_m) * 32;
    const int j0 = (local / tiles_m) * 32;
    __shared__ double2 sA[16][33];
    __shared__ double2 sB[16][33];
    const int tx = threadIdx.x % 32;
    const int ty = threadIdx.x / 32;
    double2 acc[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[c] = make_double2(0, 0);
    for (int k0 = 0; k0 < job.k; k0 += 16) {
        for (int idx = threadIdx.x; idx < 16 * 32; idx += 256) {
            const int kk = idx / 32, r = idx % 32;
            const int kg = k0 + kk;
            sA[kk][r] = (kg < job.k && i0 + r < job.m) ? load_op(job.A, job.lda, job.opA, i0 + r, kg)
                                                      : make_double2(0, 0);
            // op(B)(kg, j0 + r)
            sB[kk][r] = (kg < job.k && j0 + r < job.n) ? load_op(job.B, job.ldb, job.opB, kg, j0 + r)
                                                      : make_double2(0, 0);
        }
        __syncthreads();
#pragma unroll 4
        for (int kk = 0; kk < 16; ++kk) {
            const double2 a = sA[kk][tx];
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const double2 b = sB[kk][ty * 4 + c];
                acc[c].x = fma(a.x, b.x, fma(-a.y, b.y, acc[c].x));
                acc[c].y = fma(a.x, b.y, fma(a.y, b.x, acc[c].y));
            }
        }
        __syncthreads();
    }
    const int i = i0 + tx;
    if (i < job.m) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int j = j0 + ty * 4 + c;
            if (j < job.n) {
                double2 *cp = job.C + i + (size_t)j * job.ldc;
                double2 v = make_double2(job.alpha.x * acc[c].x - job.alpha.y * acc[c].y,
                                         job.alpha.x * acc[c].y + job.alpha.y * acc[c].x);
                if (job.beta.x != 0.0 || job.beta.y != 0.0) {
                    const double2 o = *cp;
                    v.x += job.beta.x * o.x - job.beta.y * o.y;
                    v.y += job.beta.x * o.y + job.beta.y * o.x;
                }
                *cp = v;
            }
        }
    }
}

int zgemm_tiles(const ZgemmJob &j) { return ((j.m + 31) / 32) * ((j.n + 31) / 32); }

int launch_zgemm(const std::vector<ZgemmJob> &jobs, cudaStream_t stream, DevBuf &scratch) {
    const int nj = (int)jobs.size();
    if (nj == 0) return PSKEL_OK;
    std::vector<int> prefix(nj + 1, 0);
    for (int i = 0; i < nj; ++i) prefix[i + 1] = prefix[i] + zgemm_tiles(jobs[i]);
    const int total = prefix[nj];
    if (total == 0) return PSKEL_OK;
    const size_t jb = sizeof(ZgemmJob) * nj;
    const size_t pb = sizeof(int) * (nj + 1);
    PSKEL_TRY(scratch.reserve(jb + pb + 256));
    char *base = scratch.as<char>();
    ZgemmJob *d_jobs = reinterpret_cast<ZgemmJob *>(base);
    int *d_prefix = reinterpret_cast<int *>(base + ((jb + 255) & ~size_t(255)));
    PSKEL_CUDA(cudaMemcpyAsync(d_jobs, jobs.data(), jb, cudaMemcpyHostToDevice, stream));
    PSKEL_CUDA(cudaMemcpyAsync(d_prefix, prefix.data(), pb, cudaMemcpyHostToDevice, stream));
    zgemm_kernel<<<total, 256, 0, stream>>>(d_jobs, d_prefix, nj);
    PSKEL_LAUNCHED(1);
    return PSKEL_OK;
}

int launch_zgemm_device(const ZgemmJob *d_jobs, const int *d_prefix, int njobs, int total_tiles,
                        cudaStream_t stream) {
    if (total_tiles <= 0) return PSKEL_OK;
    zgemm_kernel<<<total_tiles, 256, 0, stream>>>(d_jobs, d_prefix, njobs);
    PSKEL_LAUNCHED(1);
    return PSKEL_OK;
}

}  // namespace pskel
