// pskel_pinv_noalloc: the truncated pseudo-inverse of one small complex matrix that performs
// no device allocation at all.
//
// Why it exists: some callers cannot call cudaMalloc. They may run inside a host framework
// that owns the device memory through its own pool and forbids allocations outside it, or in
// a latency-critical loop where cudaMalloc/cudaFree are not allowed because they can block on
// or synchronise the device. The other entry points of this library allocate (and pool)
// their workspace; this one keeps its scratch - the working copy of A, the Jacobi rotations,
// the singular values, their order and the job descriptors - in one file-scope device array
// of kNoAllocScratchBytes (256 KiB). Every GPU that loads the library holds that array until
// the process exits.
//
// Limits and behaviour:
//  * m, n <= kNoAllocMaxDim (64); larger sizes are rejected with PSKEL_ERR_ARG.
//  * The caller passes device buffers for the input A (m x n) and the output P (n x m), and
//    optionally sigma (min(m, n), sorted descending) and rank; the stream may be NULL.
//  * The first call on a device looks up the device address of the scratch array
//    (cudaGetSymbolAddress, with that device current) and sets the kernel attributes; make
//    that first call before any stream capture.
//  * The call reads the convergence status back and waits for its stream (see below), which
//    a stream capture does not allow: on a stream that is being captured it returns
//    PSKEL_ERR_STATE before doing anything, so the caller's capture stays intact.
//  * All calls share the array, and it keeps the contents of the last call; everything the
//    kernels read is written by the same call before it is read. Calls whose work overlaps
//    on the GPU (other streams or host threads) race on the array: serialise them.
//  * The call waits for its stream before returning, so that it can report the Jacobi
//    convergence status.
#include <cfloat>

#include "pskel_internal.cuh"

namespace pskel {

constexpr int kNoAllocMaxDim = 64;
constexpr size_t kNoAllocScratchBytes = 256 * 1024;

// The scratch: every call of pskel_pinv_noalloc works in this array.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

struct NoAllocLayout {
    // byte offsets inside g_noalloc_scratch
    static constexpr size_t mat = (size_t)kNoAllocMaxDim * kNoAllocMaxDim * sizeof(double2);
    static constexpr size_t AV = 0;
    static constexpr size_t V = AV + mat;
    static constexpr size_t Pt = V + mat;
    static constexpr size_t sigma = Pt + mat;
    static constexpr size_t perm = sigma + kNoAllocMaxDim * sizeof(double);
    static constexpr size_t rank = perm + kNoAllocMaxDim * sizeof(int);
    static constexpr size_t idx = rank + 256;
    static constexpr size_t svd = idx + 256;
    static constexpr size_t pinv = svd + 256;
    static constexpr size_t end = pinv + 256;
};
static_assert(NoAllocLayout::end <= kNoAllocScratchBytes, "no-alloc scratch too small");
static_assert(sizeof(SvdJob) <= 256 && sizeof(PinvJob) <= 256, "job descriptors exceed slots");

// Writes the job descriptors and the working copy of A (or A^H when m < n) into the scratch.
__global__ void noalloc_setup_kernel(unsigned char *base, const double2 *A, int M, int N,
                                     double tau, int relative) {
    const bool tr = M < N;
    const int m = tr ? N : M, n = tr ? M : N;
    double2 *AV = reinterpret_cast<double2 *>(base + NoAllocLayout::AV);
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < M * N; idx += gridDim.x * blockDim.x) {
        const int i = idx % M, j = idx / M;
        const double2 v = A[idx];
        if (!tr) AV[i + j * m] = v;
        else AV[j + i * m] = make_double2(v.x, -v.y);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        SvdJob *sj = reinterpret_cast<SvdJob *>(base + NoAllocLayout::svd);
        sj->A = AV;
        sj->V = reinterpret_cast<double2 *>(base + NoAllocLayout::V);
        sj->sigma = reinterpret_cast<double *>(base + NoAllocLayout::sigma);
        sj->perm = reinterpret_cast<int *>(base + NoAllocLayout::perm);
        sj->m = m;
        sj->n = n;
        sj->status = PSKEL_ERR_NOCONV;  // overwritten by the SVD kernel
        sj->sweeps = 0;
        sj->trunc = 0.0;
        *reinterpret_cast<int *>(base + NoAllocLayout::idx) = 0;
        *reinterpret_cast<int *>(base + NoAllocLayout::rank) = 0;
        PinvJob *pj = reinterpret_cast<PinvJob *>(base + NoAllocLayout::pinv);
        pj->AV = AV;
        pj->V = sj->V;
        pj->sigma = sj->sigma;
        pj->P = reinterpret_cast<double2 *>(base + NoAllocLayout::Pt);  // n x m
        pj->rank = reinterpret_cast<int *>(base + NoAllocLayout::rank);
        pj->m = m;
        pj->n = n;
        pj->tau = tau;
        pj->relative = relative;
    }
}

// P (N x M) from the pinv of the working matrix, sorted singular values and the rank.
__global__ void noalloc_finish_kernel(const unsigned char *base, int M, int N, double2 *P,
                                      double *sigma_out, int *rank_out) {
    const bool tr = M < N;
    const int n = tr ? M : N;  // working matrix (tr ? N : M) x n, its pinv Pt has n rows
    const double2 *Pt = reinterpret_cast<const double2 *>(base + NoAllocLayout::Pt);
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < M * N; idx += gridDim.x * blockDim.x) {
        const int a = idx % N, b = idx / N;  // P(a, b), a < N, b < M
        double2 v;
        if (!tr) {
            v = Pt[a + b * n];
        } else {  // pinv(A) = pinv(A^H)^H: P(a, b) = conj(Pt(b, a)), Pt is M x N here
            const double2 w = Pt[b + a * n];
            v = make_double2(w.x, -w.y);
        }
        P[a + (size_t)b * N] = v;
    }
    if (blockIdx.x == 0) {
        const double *sg = reinterpret_cast<const double *>(base + NoAllocLayout::sigma);
        const int *pm = reinterpret_cast<const int *>(base + NoAllocLayout::perm);
        if (sigma_out)
            for (int r = threadIdx.x; r < n; r += blockDim.x) sigma_out[r] = sg[pm[r]];
        if (rank_out && threadIdx.x == 0) *rank_out = *reinterpret_cast<const int *>(base + NoAllocLayout::rank);
    }
}

namespace {
unsigned char *g_scratch_addr[kMaxDevices] = {};
std::mutex g_setup_mu;

int noalloc_setup_device(int dev, unsigned char **out) {
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        PSKEL_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        // the resident SVD kernel needs (m n + n n) complex doubles of shared memory
        PSKEL_TRY(svd_resident_attr());
        g_scratch_addr[dev] = static_cast<unsigned char *>(p);
    }
    *out = g_scratch_addr[dev];
    return PSKEL_OK;
}
}  // namespace

}  // namespace pskel

using namespace pskel;

extern "C" int pskel_pinv_noalloc(const pskel_c128 *A, int M, int N, double tau, int relative,
                                  pskel_c128 *P, double *sigma, int *rank, void *stream) {
    if (!A || !P || M <= 0 || N <= 0 || tau < 0) {
        set_error(PSKEL_ERR_ARG, "pinv_noalloc: null buffer or bad size (M=%d N=%d)", M, N);
        return PSKEL_ERR_ARG;
    }
    if (M > kNoAllocMaxDim || N > kNoAllocMaxDim) {
        set_error(PSKEL_ERR_ARG, "pinv_noalloc: %d x %d exceeds the fixed scratch limit of %d x %d",
                  M, N, kNoAllocMaxDim, kNoAllocMaxDim);
        return PSKEL_ERR_ARG;
    }
    int dev = 0;
    PSKEL_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error(PSKEL_ERR_ARG, "pinv_noalloc: device %d out of range", dev);
        return PSKEL_ERR_ARG;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    PSKEL_CUDA(cudaStreamIsCapturing(s, &cap));
    if (cap != cudaStreamCaptureStatusNone) {
        set_error(PSKEL_ERR_STATE, "pinv_noalloc: the stream is being captured; the call waits "
                                   "for its stream to read the convergence status");
        return PSKEL_ERR_STATE;
    }
    unsigned char *base = nullptr;
    PSKEL_TRY(noalloc_setup_device(dev, &base));
    const double2 *Ad = reinterpret_cast<const double2 *>(A);
    noalloc_setup_kernel<<<16, 256, 0, s>>>(base, Ad, M, N, tau, relative);
    PSKEL_LAUNCHED(1);
    const int m = M < N ? N : M, n = M < N ? M : N;
    SvdJob *sj = reinterpret_cast<SvdJob *>(base + NoAllocLayout::svd);
    const int *idx = reinterpret_cast<const int *>(base + NoAllocLayout::idx);
    PSKEL_TRY(svd_launch_single_resident(sj, idx, m, n, 60, s));
    const PinvJob *pj = reinterpret_cast<const PinvJob *>(base + NoAllocLayout::pinv);
    PSKEL_TRY(batched_pinv(pj, 1, ((n + 31) / 32) * ((m + 31) / 32), s));
    noalloc_finish_kernel<<<16, 256, 0, s>>>(base, M, N, reinterpret_cast<double2 *>(P), sigma, rank);
    PSKEL_LAUNCHED(1);
    int st[2] = {0, 0};
    PSKEL_CUDA(cudaMemcpyAsync(st, &sj->status, sizeof(st), cudaMemcpyDeviceToHost, s));
    PSKEL_CUDA(cudaStreamSynchronize(s));
    if (st[0] != PSKEL_OK) {
        set_error(PSKEL_ERR_NOCONV, "pinv_noalloc: Jacobi SVD did not converge in %d sweeps", st[1]);
        return PSKEL_ERR_NOCONV;
    }
    return PSKEL_OK;
}
