// Shared internals of libpskel_b200: status handling, device buffers, mesh records.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

#include "device_state.hpp"
#include "pskel.h"

namespace pskel {

// ------------------------------------------------------------------ errors
void set_error(int code, const char *fmt, ...);
int last_code();

#define PSKEL_CUDA(call)                                                                   \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) {                                                           \
            ::pskel::set_error(e_ == cudaErrorMemoryAllocation ? PSKEL_ERR_OOM            \
                                                               : PSKEL_ERR_CUDA,          \
                               "%s:%d %s: %s", __FILE__, __LINE__, #call,                  \
                               cudaGetErrorString(e_));                                    \
            return e_ == cudaErrorMemoryAllocation ? PSKEL_ERR_OOM : PSKEL_ERR_CUDA;       \
        }                                                                                  \
    } while (0)

#define PSKEL_TRY(expr)                      \
    do {                                     \
        int s_ = (expr);                     \
        if (s_ != PSKEL_OK) return s_;       \
    } while (0)

// ------------------------------------------------------------------ device buffer
// Grow-only device allocation reused across calls (no cudaMalloc on the steady path).
struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    int reserve(size_t want) {
        if (want <= bytes) return PSKEL_OK;
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
        size_t sz = want < 256 ? 256 : want;
        sz = (sz + 255) & ~size_t(255);
        PSKEL_CUDA(cudaMalloc(&ptr, sz));
        bytes = sz;
        return PSKEL_OK;
    }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    template <typename T> T *as() const { return static_cast<T *>(ptr); }
};

// Page-locked host buffer: job tables are packed here and uploaded with one asynchronous copy
// (a pageable source is staged by the driver and blocks the host for the transfer). The owner
// must not repack it before the stream has consumed the previous upload.
struct PinnedBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    int reserve(size_t want) {
        if (want <= bytes) return PSKEL_OK;
        if (ptr) cudaFreeHost(ptr);
        ptr = nullptr;
        bytes = 0;
        size_t sz = want < 4096 ? 4096 : want;
        sz = (sz + 4095) & ~size_t(4095);
        PSKEL_CUDA(cudaHostAlloc(&ptr, sz, cudaHostAllocDefault));
        bytes = sz;
        return PSKEL_OK;
    }
    void release() {
        if (ptr) cudaFreeHost(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    template <typename T> T *as() const { return static_cast<T *>(ptr); }
};

// ------------------------------------------------------------------ mesh records
// Per-RWG quadrature record: for the 2Q points of the basis (Q on T+, then Q on T-), seven
// fields stored field-major: x[2Q] y[2Q] z[2Q] ux[2Q] uy[2Q] uz[2Q] d[2Q], where
//   u = w_p * (l/2) * rho(r_p),  rho = s (r_p - v_opp),  d = w_p * s * l,  s = +1 (T+), -1 (T-)
// so that Z_mn = eta/(4 pi) * sum_{p,q} A_pq (sin kR + j cos kR) / R with
//   A_pq = d_p e_q / k - k u_p . v_q.
// The record stride is padded to an odd number of doubles.
__host__ __device__ constexpr int rec_points(int q) { return 2 * q; }
__host__ __device__ constexpr int rec_stride(int q) { return (7 * 2 * q) | 1; }

struct MeshRecords {
    int q = 0;
    DevBuf f64;  // ne * rec_stride(q) doubles
    DevBuf tri;  // nt * tri_stride(q) doubles: the q points (x, y, z) of each triangle, then
                 // its centroid (x, y, z)
};
__host__ __device__ constexpr int tri_stride(int q) { return 3 * (q + 1); }

struct DevMesh {
    int ne = 0, nt = 0, nv = 0;
    DevBuf vertex, topol, edges, ln, cent;  // reference arrays as doubles
    MeshRecords rec1, rec7;                 // Q = 1 and Q = 7 records (built on demand)
    MeshRecords &records(int q) { return q == 1 ? rec1 : rec7; }
};

// Weights of the q-point triangle rule (q = 1: {1}; q = 7: the 7-point rule), summing to 1.
void quadrature_weights(int q, double *w);

// Build (or rebuild) the Q-point records of a mesh whose raw arrays are on the device.
int build_records(DevMesh &mesh, int q, cudaStream_t stream, int *d_flag);

// Upload the raw reference arrays (host, column-major doubles) into mesh.
int upload_mesh_arrays(DevMesh &mesh, const double *vertex, int nv, const double *topol, int nt,
                       const double *edges, int ne, const double *ln, const double *cent,
                       cudaStream_t stream);

// ------------------------------------------------------------------ fill
// One fill job: Z(rows, cols) -> out (column-major, leading dimension ld). rows/cols are
// 0-based RWG ids in device memory.
struct FillJob {
    const int *rows;
    const int *cols;
    void *out;
    int nr, nc, ld;
    int trans;  // 1: store Z(rows, cols) transposed, out[j + i * ld] (Galerkin symmetry lets a
                // caller fill Z(a, b) as the transpose of Z(b, a) with the long side on rows)
};

constexpr int kTriFillCols = 16;        // most columns per CTA tile (variants 4, 8, 16)
constexpr int kTriFillColsDefault = 8;
constexpr int kTriFillMaxRowsDefaultForParams = 512;

struct FillParams {
    double k, eta;
    double r_near;     // > 0: flag triangle pairs whose centroids are closer than this
    int q_test, q_src;
    int precision;     // PSKEL_C128 / PSKEL_C64
    int split;         // 0: two rows per thread (default kernel); 1, 2, 4: lanes per entry
    int tri_cols = kTriFillColsDefault;  // columns per CTA of the triangle-moment fill (4, 8, 16)
    int geom32 = 0;    // complex-FP32 triangle-moment fill: FP32 pair geometry from item offsets
    int max_rows = kTriFillMaxRowsDefaultForParams;  // largest group in a triangle-moment launch
    bool persistent = true;  // grid of SM count x occupancy striding over the tiles; false: one
                             // CTA per tile (CTAs retire continually, so kernels on other streams
                             // can take their place)
    const int *const *gates = nullptr;  // non-null: per job, a device flag; the tiles of a job
                                        // whose flag is 0 do nothing (jobs planned ahead whose
                                        // use is decided on the device)
};

// Launch the batched fill over jobs (device array) with tile prefix offsets computed on the
// host (tile_prefix has njobs+1 entries, device). flags[0] receives PSKEL near-field / range
// bits. Returns PSKEL_OK or an error.
int launch_fill(const DevMesh &mesh, const FillParams &p, const FillJob *d_jobs,
                const int *d_tile_prefix, int njobs, int total_tiles, int *d_flags,
                cudaStream_t stream);
int fill_tile_shape(int precision, int q, int split, int *tm, int *tn);

// Near-field rule (csrc/near.cu): radii of the reference's element routine and the rule of a
// side outside its radius (1 = centroid, 7 = 7-point).
struct NearRadii {
    double rinteg_s = 0.0, ranal_s = 0.0, rinteg_f = 0.0;
    int q_far = 1;
};
// Complex-FP64 fill of the jobs (host list) with the near-field rule, one thread per entry;
// the same-triangle moments go to mom (8 double2 per triangle), for every triangle or only for
// the triangles of the jobs' rows. patch: only the entries with a same-triangle pair or a pair
// inside a radius are written (the caller filled the rest with the far rule). flags bit 2 / 4:
// RWG / triangle id out of range.
int near_fill_jobs(const DevMesh &mesh, const NearRadii &r, double k, double eta,
                   const std::vector<FillJob> &jobs, DevBuf &scratch, DevBuf &mom, int *d_flags,
                   cudaStream_t stream, bool all_triangles, bool patch);

// Triangle-moment fill of Z(group, cols) for a group of RWG functions whose triangle list and
// triangle -> (RWG, side) adjacency are known (see tri_fill_kernel in fill.cu).
struct GroupFillJob {
    const int *rows;  // global RWG ids of the group (m)
    const int *tris;  // global triangle ids touched by the group (nt)
    const int *adj;   // 3 per triangle: 2 * local RWG index + side (0: T+, 1: T-), or -1
    const int *cols;  // global RWG ids of the columns (nc)
    void *out;
    int m, nt, nc, ld, trans;
    int tc;           // columns per CTA tile for this job (<= the launch's tile width)
    const double *use;  // 4 doubles per (triangle, adjacency slot): the RWG's free vertex minus
                        // the triangle centroid (x, y, z) and the signed edge length s l; null:
                        // looked up in the mesh arrays
};
constexpr int kTriFillMaxRows = 512;  // largest group the triangle-moment fill accepts
// Columns per tile for a job of nt triangles: the width in [4, max_cols] whose (triangle, column)
// item count fills the 256 threads of a CTA best (the last round of items is the idle part),
// the widest among equals. max_cols < 4 returns max_cols.
inline int tri_tile_cols(int nt, int max_cols) {
    constexpr int threads = 256;
    if (max_cols < 4) return max_cols < 1 ? 1 : max_cols;
    int best = max_cols;
    double best_eff = -1.0;
    for (int c = max_cols; c >= 4; --c) {
        const long long items = (long long)nt * c;
        const long long slots = (items + threads - 1) / threads * threads;
        const double eff = (double)items / (double)slots;
        if (eff > best_eff + 1e-9) {
            best_eff = eff;
            best = c;
        }
    }
    return best;
}
int launch_tri_fill(const DevMesh &mesh, const FillParams &p, const GroupFillJob *d_jobs,
                    const int *d_tile_prefix, int njobs, int total_tiles, cudaStream_t stream);

// Convert 1-based double ids to 0-based int32 with a range check (flags bit 1 on error).
int launch_ids_from_double(const double *d_in, int *d_out, int n, int limit, int *d_flags,
                           cudaStream_t stream);
int launch_ids_from_int64(const int64_t *d_in, int *d_out, int n, int limit, int *d_flags,
                          cudaStream_t stream);

// ------------------------------------------------------------------ Jacobi SVD / pinv
// Batched one-sided Jacobi SVD of complex128 matrices A_b (m_b x n_b, column-major, lda = m_b)
// with m_b >= n_b. Work is in place: on return A_b holds A_b V_b (orthogonal columns) and V_b
// (n_b x n_b) the accumulated rotations.
struct SvdJob {
    double2 *A;      // m x n, overwritten by A V
    double2 *V;      // n x n
    double *sigma;   // n, singular values in column order (unsorted)
    int *perm;       // n, column indices sorted by decreasing sigma (may be null)
    int m, n;
    int status;      // written by the kernel: 0 converged, PSKEL_ERR_NOCONV otherwise
    int sweeps;
    // > 0 (resident kernel only): truncated SVD. The pivoted QR stops at the first k whose
    // trailing block has Frobenius norm <= trunc; the k singular triplets of the leading rows
    // are returned and the other columns of A V, V and sigma are zero. Every singular value
    // moves by at most trunc.
    double trunc;
};

// Run the SVD of every job to convergence (max_sweeps cap). jobs is a DEVICE array; the host
// copy is used for sizes. Returns PSKEL_OK even if some job failed to converge (their status
// field says so).
int batched_svd(SvdJob *d_jobs, const std::vector<SvdJob> &h_jobs, int max_sweeps,
                cudaStream_t stream, DevBuf &scratch);

// The same work as a host plan (job order: resident jobs by size class, then blocked ones) and
// launches from device tables, so the launches can be captured in a CUDA graph.
struct SvdPlan {
    struct Cls {
        int off, count;  // range of the index map
        size_t smem;     // dynamic shared memory of the class
        int threads;
    };
    std::vector<int> idx;  // job order
    std::vector<Cls> res;  // resident classes
    int blk_off = 0, blk_count = 0;
};
int svd_plan(const std::vector<SvdJob> &h_jobs, SvdPlan &plan);
int svd_plan(const SvdJob *h_jobs, int nj, SvdPlan &plan);
// Side streams for the size-class launches of one SVD plan: the classes are independent, so
// they run concurrently (fork on `fork`, join through `join`); graph capture follows the events.
constexpr int kSvdAux = 4;
struct SvdStreams {
    cudaStream_t aux[kSvdAux] = {};
    cudaEvent_t fork = nullptr, join[kSvdAux] = {};
    bool ready = false;
};
int svd_streams_create(SvdStreams &p);
void svd_streams_destroy(SvdStreams &p);
int svd_launch(SvdJob *d_jobs, const int *d_idx, const SvdPlan &plan, int max_sweeps,
               cudaStream_t stream, const SvdStreams *par = nullptr);
// One resident job (m x n fits in shared memory) whose index map entry is d_idx0[0].
int svd_launch_single_resident(SvdJob *d_job, const int *d_idx0, int m, int n, int max_sweeps,
                               cudaStream_t stream);
// Shared-memory limits of the SVD kernels on the current device (set once per device).
int svd_resident_attr();

// pinv of each job after batched_svd: P_b (n_b x m_b) = V diag(1/sigma^2) (A V)^H over the
// kept columns; rank_b receives the count kept. thr_b = tau (absolute) or tau * sigma_max.
struct PinvJob {
    const double2 *AV;
    const double2 *V;
    const double *sigma;
    double2 *P;      // n x m output, ld = n
    int *rank;
    int m, n;
    double tau;
    int relative;
};
int batched_pinv(const PinvJob *d_jobs, int njobs, int max_n, cudaStream_t stream);

// Householder QR of m x n complex matrices (m >= n), in place: the reflector tails below the
// diagonal of A, v(0) and coef = 2 / |v|^2 of each reflector in v0 / coef, R (n x n, zero below
// the diagonal) in R. Job tables go through scratch.
struct QrJob {
    double2 *A;
    double2 *R;
    double2 *v0;
    double *coef;
    int m, n;
};
int batched_qr(const std::vector<QrJob> &h_jobs, cudaStream_t stream, DevBuf &scratch);

// Y (m x kcols, ld ldy) = Q [Z; 0] for the Q of a batched_qr job (reflectors A, v0, coef; Z is
// n x kcols, ld ldz); kcols = min(k, *kp) when kp is given (a device count).
struct ApplyQJob {
    const double2 *A;
    const double2 *v0;
    const double *coef;
    int m, n;
    const double2 *Z;
    int ldz;
    double2 *Y;
    int ldy;
    int k;
    const int *kp;
};
int batched_apply_q(const std::vector<ApplyQJob> &h_jobs, cudaStream_t stream, DevBuf &scratch);

// ------------------------------------------------------------------ small dense helpers
// y = C (U (R x)) and the successive-estimate error of the reference (complex128).
int cur_matvec_error(const double2 *C, const double2 *U, const double2 *R, const double2 *x,
                     const double2 *y_old, double2 *y_new, int m, int r, int n, double *err,
                     cudaStream_t stream, DevBuf &scratch);

// ------------------------------------------------------------------ device properties
// SM count of the current device.
int sm_count();

// Raises the dynamic-shared-memory limit of a kernel on the CURRENT device to at least `bytes`
// (the attribute is per device; set once per kernel, device and size; thread-safe).
int ensure_smem_attr(const void *func, size_t bytes);
template <typename K>
int ensure_smem_attr(K *kern, size_t bytes) {
    return ensure_smem_attr(reinterpret_cast<const void *>(kern), bytes);
}

// Count of kernels launched by the library (reported by pskel_kernel_launches).
void count_launch(long long n = 1);
long long launches_so_far();
// After each kernel launch: count it and surface a launch error.
#define PSKEL_LAUNCHED(n)                 \
    do {                                  \
        ::pskel::count_launch(n);         \
        PSKEL_CUDA(cudaGetLastError());   \
    } while (0)

}  // namespace pskel
