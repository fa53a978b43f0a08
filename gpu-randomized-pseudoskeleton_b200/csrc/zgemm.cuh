// Batched complex FP64 GEMM (see zgemm.cu).
#pragma once
#include <vector>

#include "pskel_internal.cuh"

namespace pskel {

enum { ZOP_N = 0, ZOP_C = 1, ZOP_T = 2 };

// C (m x n, ldc) = alpha op(A) (m x k) op(B) (k x n) + beta C
struct ZgemmJob {
    const double2 *A;
    const double2 *B;
    double2 *C;
    int m, n, k;
    int lda, ldb, ldc;
    int opA, opB;
    double2 alpha, beta;
};

inline ZgemmJob zjob(const double2 *A, int lda, int opA, const double2 *B, int ldb, int opB,
                     double2 *C, int ldc, int m, int n, int k) {
    ZgemmJob j;
    j.A = A; j.B = B; j.C = C;
    j.m = m; j.n = n; j.k = k;
    j.lda = lda; j.ldb = ldb; j.ldc = ldc;
    j.opA = opA; j.opB = opB;
    j.alpha = make_double2(1.0, 0.0);
    j.beta = make_double2(0.0, 0.0);
    return j;
}

int zgemm_tiles(const ZgemmJob &j);
// Uploads the job list to scratch and launches one kernel over every tile of every job.
int launch_zgemm(const std::vector<ZgemmJob> &jobs, cudaStream_t stream, DevBuf &scratch);
int launch_zgemm_device(const ZgemmJob *d_jobs, const int *d_prefix, int njobs, int total_tiles,
                        cudaStream_t stream);

}  // namespace pskel
