// Reference-named C entry points (drop-ins for functionsExternal_cuda.so and
// functions_cur_external_cuda.so). Each one keeps the reference's argument list, host-pointer
// convention and return type; the work runs on the library's own kernels (fill.cu, jacobi.cu,
// zgemm.cu) with device buffers pooled across calls instead of cudaMalloc/cudaFree per call.
#include <cmath>
#include <limits>
#include <mutex>

#include "pskel_internal.cuh"
#include "zgemm.cuh"

namespace pskel {
namespace {

struct LegacyCtx {
    bool init = false;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    DevMesh mesh;
    DevBuf flags, ids_raw, ids, jobs, out, work, scratch, scratch2;
    DevBuf near_jobs, near_mom;  // near-field fill: job table and same-triangle moments
    std::mutex mu;
};

// One context per device ordinal: the reference entry points run on whichever device is
// current when they are called, and streams, events and buffers belong to one device.
LegacyCtx *ctx() {
    static PerDevice<LegacyCtx> contexts;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        set_error(PSKEL_ERR_CUDA, "cudaGetDevice failed");
        return nullptr;
    }
    LegacyCtx *c = contexts.get(dev);
    if (!c) set_error(PSKEL_ERR_ARG, "device ordinal %d beyond %d", dev, kMaxDevices);
    return c;
}

int ensure_init(LegacyCtx &c) {
    if (c.init) return PSKEL_OK;
    PSKEL_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
    PSKEL_CUDA(cudaEventCreate(&c.ev0));
    PSKEL_CUDA(cudaEventCreate(&c.ev1));
    PSKEL_TRY(c.flags.reserve(256));
    c.init = true;
    return PSKEL_OK;
}

const double kNaN = std::numeric_limits<double>::quiet_NaN();

// Upload the mesh and build Q = 1 records (the reference's centroid rule).
int prepare_mesh(LegacyCtx &c, double *vertex, int rows_vertex, int cols_vertex, double *topol,
                 int rows_topol, int cols_topol, double *edges, int rows_edges, int cols_edges,
                 double *ln, int n_ln, double *cent, int rows_cent, int cols_cent) {
    if (rows_vertex != 3 || rows_topol != 3 || rows_edges != 4 || rows_cent != 3 ||
        cols_edges != n_ln || cols_cent != cols_topol) {
        set_error(PSKEL_ERR_ARG,
                  "mesh shape: vertex %dx%d topol %dx%d edges %dx%d ln %d cent %dx%d",
                  rows_vertex, cols_vertex, rows_topol, cols_topol, rows_edges, cols_edges,
                  n_ln, rows_cent, cols_cent);
        return PSKEL_ERR_ARG;
    }
    PSKEL_TRY(upload_mesh_arrays(c.mesh, vertex, cols_vertex, topol, cols_topol, edges,
                                 cols_edges, ln, cent, c.stream));
    PSKEL_CUDA(cudaMemsetAsync(c.flags.ptr, 0, 256, c.stream));
    PSKEL_TRY(build_records(c.mesh, 1, c.stream, c.flags.as<int>()));
    return PSKEL_OK;
}

// 1-based double id lists -> 0-based int32 on the device. Lists are concatenated into ids.
int upload_ids(LegacyCtx &c, const double *const *lists, const int *lens, int nlists, int limit,
               int **d_out) {
    size_t total = 0;
    for (int i = 0; i < nlists; ++i) total += lens[i];
    PSKEL_TRY(c.ids_raw.reserve(sizeof(double) * (total + 1)));
    PSKEL_TRY(c.ids.reserve(sizeof(int) * (total + 1)));
    size_t off = 0;
    for (int i = 0; i < nlists; ++i) {
        if (lens[i] > 0) {
            if (!lists[i]) {
                set_error(PSKEL_ERR_ARG, "null id list");
                return PSKEL_ERR_ARG;
            }
            PSKEL_CUDA(cudaMemcpyAsync(c.ids_raw.as<double>() + off, lists[i],
                                       sizeof(double) * lens[i], cudaMemcpyHostToDevice,
                                       c.stream));
        }
        d_out[i] = c.ids.as<int>() + off;
        off += lens[i];
    }
    PSKEL_TRY(launch_ids_from_double(c.ids_raw.as<double>(), c.ids.as<int>(), (int)total, limit,
                                     c.flags.as<int>(), c.stream));
    return PSKEL_OK;
}

// Fill the jobs with the reference's element routine semantics: the centroid-rule kernel first,
// flagging any triangle pair closer than the largest radius (and every same-triangle pair, whose
// centroid distance is 0); if one is flagged, the whole request is refilled by the near-field
// kernel (4-point rules, exact static 1/R, same-triangle term), so far-only requests keep the
// fast path. Synchronises the stream when flagging is possible.
int fill_jobs(LegacyCtx &c, const std::vector<FillJob> &jobs, double k, double eta,
              const NearRadii &radii) {
    int tm, tn;
    fill_tile_shape(PSKEL_C128, 1, 0, &tm, &tn);
    std::vector<int> prefix(jobs.size() + 1, 0);
    for (size_t i = 0; i < jobs.size(); ++i)
        prefix[i + 1] = prefix[i] + ((jobs[i].nr + tm - 1) / tm) * ((jobs[i].nc + tn - 1) / tn);
    const size_t jb = sizeof(FillJob) * jobs.size();
    PSKEL_TRY(c.jobs.reserve(jb + 256 + sizeof(int) * prefix.size()));
    FillJob *d_jobs = c.jobs.as<FillJob>();
    int *d_prefix = reinterpret_cast<int *>(c.jobs.as<char>() + ((jb + 255) & ~size_t(255)));
    PSKEL_CUDA(cudaMemcpyAsync(d_jobs, jobs.data(), jb, cudaMemcpyHostToDevice, c.stream));
    PSKEL_CUDA(cudaMemcpyAsync(d_prefix, prefix.data(), sizeof(int) * prefix.size(),
                               cudaMemcpyHostToDevice, c.stream));
    double r = radii.rinteg_s;
    if (radii.ranal_s > r) r = radii.ranal_s;
    if (radii.rinteg_f > r) r = radii.rinteg_f;
    FillParams p;
    p.k = k;
    p.eta = eta;
    p.r_near = r > 1e-150 ? r : 1e-150;  // > 0: same-triangle pairs (distance 0) are flagged too
    p.q_test = p.q_src = 1;
    p.precision = PSKEL_C128;
    p.split = 0;
    PSKEL_TRY(launch_fill(c.mesh, p, d_jobs, d_prefix, (int)jobs.size(), prefix.back(),
                          c.flags.as<int>(), c.stream));
    int h = 0;
    PSKEL_CUDA(cudaMemcpyAsync(&h, c.flags.ptr, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    PSKEL_CUDA(cudaStreamSynchronize(c.stream));
    if (!(h & 1) || (h & 6)) return PSKEL_OK;  // far only, or a range error (check_flags)
    PSKEL_CUDA(cudaMemsetAsync(c.flags.ptr, 0, sizeof(int), c.stream));
    return near_fill_jobs(c.mesh, radii, k, eta, jobs, c.near_jobs, c.near_mom, c.flags.as<int>(),
                          c.stream, false, false);
}

// Read the flag word after the stream drains; maps bits to statuses.
int check_flags(LegacyCtx &c) {
    int h = 0;
    PSKEL_CUDA(cudaMemcpyAsync(&h, c.flags.ptr, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    PSKEL_CUDA(cudaStreamSynchronize(c.stream));
    if (h & 6) {
        set_error(PSKEL_ERR_RANGE, "an RWG, triangle or vertex id is out of range");
        return PSKEL_ERR_RANGE;
    }
    return PSKEL_OK;
}

NearRadii radii_of(double Rinteg_s, double Ranal_s, double Rinteg_f) {
    NearRadii r;
    r.rinteg_s = Rinteg_s;
    r.ranal_s = Ranal_s;
    r.rinteg_f = Rinteg_f;
    r.q_far = 1;
    return r;
}

int check_field(int field) {
    if (field != 1) {
        set_error(PSKEL_ERR_UNSUPPORTED, "field=%d: only EFIE (field=1) is implemented", field);
        return PSKEL_ERR_UNSUPPORTED;
    }
    return PSKEL_OK;
}

// Dense fill Z(r1, r2) into c.out; returns status and the kernel ms.
int dense_fill(LegacyCtx &c, int field, double k, double eta, double Rinteg_s, double Ranal_s,
               double Rinteg_f, int *r1, int *r2, double *vertex, double *topol, double *edges,
               double *ln, double *cent, int N, int n_r1, int n_r2, int rows_vertex,
               int cols_vertex, int rows_topol, int cols_topol, int rows_edges, int cols_edges,
               int n_ln, int rows_cent, int cols_cent, float *ms) {
    PSKEL_TRY(check_field(field));
    if (n_r1 < 0 || n_r2 < 0 || N != cols_edges) {
        set_error(PSKEL_ERR_ARG, "sizes: n_r1=%d n_r2=%d N=%d edges=%d", n_r1, n_r2, N, cols_edges);
        return PSKEL_ERR_ARG;
    }
    PSKEL_TRY(ensure_init(c));
    PSKEL_TRY(prepare_mesh(c, vertex, rows_vertex, cols_vertex, topol, rows_topol, cols_topol,
                           edges, rows_edges, cols_edges, ln, n_ln, cent, rows_cent, cols_cent));
    const double *lists[2] = {reinterpret_cast<double *>(r1), reinterpret_cast<double *>(r2)};
    const int lens[2] = {n_r1, n_r2};
    int *d_ids[2];
    PSKEL_TRY(upload_ids(c, lists, lens, 2, N, d_ids));
    PSKEL_TRY(c.out.reserve(sizeof(double2) * ((size_t)n_r1 * n_r2 + 1)));
    std::vector<FillJob> jobs(1);
    jobs[0] = FillJob{d_ids[0], d_ids[1], c.out.ptr, n_r1, n_r2, n_r1, 0};
    PSKEL_CUDA(cudaEventRecord(c.ev0, c.stream));
    if ((size_t)n_r1 * n_r2 > 0) PSKEL_TRY(fill_jobs(c, jobs, k, eta, radii_of(Rinteg_s, Ranal_s, Rinteg_f)));
    PSKEL_CUDA(cudaEventRecord(c.ev1, c.stream));
    PSKEL_TRY(check_flags(c));
    PSKEL_CUDA(cudaEventElapsedTime(ms, c.ev0, c.ev1));
    return PSKEL_OK;
}

}  // namespace
}  // namespace pskel

using namespace pskel;

extern "C" double impedance_matrix_cuda_elbyel4(
    pskel_c128 *Ztotal, int field, double k, double eta, double Rinteg_s, double Ranal_s,
    double Rinteg_f, int cor_solid, int flag, int *r1, int *r2, double *vertex, double *topol,
    double *trian, double *edges, double *un, double *ds, double *ln, double *cent, int N,
    int n_r1, int n_r2, int rows_vertex, int cols_vertex, int rows_topol, int cols_topol,
    int rows_trian, int cols_trian, int rows_edges, int cols_edges, int rows_un, int cols_un,
    int rows_ds, int cols_ds, int n_ln, int rows_cent, int cols_cent, int blocks_x, int blocks_y,
    int threads_x, int threads_y, int limx, int limy) {
    (void)cor_solid; (void)flag; (void)trian; (void)un; (void)ds; (void)rows_trian;
    (void)cols_trian; (void)rows_un; (void)cols_un; (void)rows_ds; (void)cols_ds;
    (void)blocks_x; (void)blocks_y; (void)threads_x; (void)threads_y; (void)limx; (void)limy;
    LegacyCtx *cp = ctx();
    if (!cp) return kNaN;
    LegacyCtx &c = *cp;
    std::lock_guard<std::mutex> lk(c.mu);
    float ms = 0;
    int st = dense_fill(c, field, k, eta, Rinteg_s, Ranal_s, Rinteg_f, r1, r2, vertex, topol,
                        edges, ln, cent, N, n_r1, n_r2, rows_vertex, cols_vertex, rows_topol,
                        cols_topol, rows_edges, cols_edges, n_ln, rows_cent, cols_cent, &ms);
    if (st == PSKEL_OK) {
        if (Ztotal && (size_t)n_r1 * n_r2 > 0 &&
            cudaMemcpy(Ztotal, c.out.ptr, sizeof(double2) * (size_t)n_r1 * n_r2,
                       cudaMemcpyDeviceToHost) != cudaSuccess) {
            set_error(PSKEL_ERR_CUDA, "D2H copy failed");
            return kNaN;
        }
    }
    return st == PSKEL_OK ? (double)ms : kNaN;
}

extern "C" int impedance_matrix_cuda_elbyel3(
    pskel_c128 *Ztotal, int field, double k, double eta, double Rinteg_s, double Ranal_s,
    double Rinteg_f, int cor_solid, int flag, int *r1, int *r2, double *vertex, double *topol,
    double *trian, double *edges, double *un, double *ds, double *ln, double *cent, int N,
    int n_r1, int n_r2, int rows_vertex, int cols_vertex, int rows_topol, int cols_topol,
    int rows_trian, int cols_trian, int rows_edges, int cols_edges, int rows_un, int cols_un,
    int rows_ds, int cols_ds, int n_ln, int rows_cent, int cols_cent, int blocks_x, int blocks_y,
    int threads_x, int threads_y, int limx, int limy) {
    const double r = impedance_matrix_cuda_elbyel4(
        Ztotal, field, k, eta, Rinteg_s, Ranal_s, Rinteg_f, cor_solid, flag, r1, r2, vertex,
        topol, trian, edges, un, ds, ln, cent, N, n_r1, n_r2, rows_vertex, cols_vertex,
        rows_topol, cols_topol, rows_trian, cols_trian, rows_edges, cols_edges, rows_un, cols_un,
        rows_ds, cols_ds, n_ln, rows_cent, cols_cent, blocks_x, blocks_y, threads_x, threads_y,
        limx, limy);
    return std::isnan(r) ? 0 : 1;
}

static int split_fill(double *Zr, double *Zi, int field, double k, double eta, double Rinteg_s,
                      double Ranal_s, double Rinteg_f, int *r1, int *r2, double *vertex,
                      double *topol, double *edges, double *ln, double *cent, int N, int n_r1,
                      int n_r2, int rows_vertex, int cols_vertex, int rows_topol, int cols_topol,
                      int rows_edges, int cols_edges, int n_ln, int rows_cent, int cols_cent) {
    LegacyCtx *cp = ctx();
    if (!cp) return 0;
    LegacyCtx &c = *cp;
    std::lock_guard<std::mutex> lk(c.mu);
    float ms = 0;
    int st = dense_fill(c, field, k, eta, Rinteg_s, Ranal_s, Rinteg_f, r1, r2, vertex, topol,
                        edges, ln, cent, N, n_r1, n_r2, rows_vertex, cols_vertex, rows_topol,
                        cols_topol, rows_edges, cols_edges, n_ln, rows_cent, cols_cent, &ms);
    if (st != PSKEL_OK) return 0;
    const size_t n = (size_t)n_r1 * n_r2;
    if (n == 0) return 1;
    std::vector<double2> h(n);
    if (cudaMemcpy(h.data(), c.out.ptr, sizeof(double2) * n, cudaMemcpyDeviceToHost) != cudaSuccess) {
        set_error(PSKEL_ERR_CUDA, "D2H copy failed");
        return 0;
    }
    for (size_t i = 0; i < n; ++i) {
        Zr[i] = h[i].x;
        Zi[i] = h[i].y;
    }
    return 1;
}

extern "C" int impedance_matrix_cuda_elbyel2(
    double *Zr, double *Zi, int field, double k, double eta, double Rinteg_s, double Ranal_s,
    double Rinteg_f, int cor_solid, int flag, int *r1, int *r2, double *vertex, double *topol,
    double *trian, double *edges, double *un, double *ds, double *ln, double *cent, int N,
    int n_r1, int n_r2, int rows_vertex, int cols_vertex, int rows_topol, int cols_topol,
    int rows_trian, int cols_trian, int rows_edges, int cols_edges, int rows_un, int cols_un,
    int rows_ds, int cols_ds, int n_ln, int rows_cent, int cols_cent, int blocks_x, int blocks_y,
    int threads_x, int threads_y, int limx, int limy) {
    (void)cor_solid; (void)flag; (void)trian; (void)un; (void)ds; (void)rows_trian;
    (void)cols_trian; (void)rows_un; (void)cols_un; (void)rows_ds; (void)cols_ds;
    (void)blocks_x; (void)blocks_y; (void)threads_x; (void)threads_y; (void)limx; (void)limy;
    return split_fill(Zr, Zi, field, k, eta, Rinteg_s, Ranal_s, Rinteg_f, r1, r2, vertex, topol,
                      edges, ln, cent, N, n_r1, n_r2, rows_vertex, cols_vertex, rows_topol,
                      cols_topol, rows_edges, cols_edges, n_ln, rows_cent, cols_cent);
}

extern "C" int cuda_cur_pure(
    double *Zr, double *Zi, int field, double k, double eta, double Rinteg_s, double Ranal_s,
    double Rinteg_f, int cor_solid, int flag, int *r1, int *r2, double *vertex, double *topol,
    double *trian, double *edges, double *un, double *ds, double *ln, double *cent,
    double *Cmat_r, double *Cmat_i, double *Umat_r, double *Umat_i, double *Rmat_r,
    double *Rmat_i, int N, int n_r1, int n_r2, int rows_vertex, int cols_vertex, int rows_topol,
    int cols_topol, int rows_trian, int cols_trian, int rows_edges, int cols_edges, int rows_un,
    int cols_un, int rows_ds, int cols_ds, int n_ln, int rows_cent, int cols_cent, int blocks_x,
    int blocks_y, int threads_x, int threads_y, int limx, int limy, double tol_compress) {
    (void)cor_solid; (void)flag; (void)trian; (void)un; (void)ds; (void)Cmat_r; (void)Cmat_i;
    (void)Umat_r; (void)Umat_i; (void)Rmat_r; (void)Rmat_i; (void)rows_trian; (void)cols_trian;
    (void)rows_un; (void)cols_un; (void)rows_ds; (void)cols_ds; (void)blocks_x; (void)blocks_y;
    (void)threads_x; (void)threads_y; (void)limx; (void)limy; (void)tol_compress;
    return split_fill(Zr, Zi, field, k, eta, Rinteg_s, Ranal_s, Rinteg_f, r1, r2, vertex, topol,
                      edges, ln, cent, N, n_r1, n_r2, rows_vertex, cols_vertex, rows_topol,
                      cols_topol, rows_edges, cols_edges, n_ln, rows_cent, cols_cent);
}

// ---------------------------------------------------------------- CUR round
namespace pskel {
namespace {

__global__ void err_kernel(const double2 *y_old, const double2 *y_new, int m, double *out) {
    __shared__ double s_d[256], s_n[256];
    double d = 0, n = 0;
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        const double2 a = y_old[i], b = y_new[i];
        const double dx = a.x - b.x, dy = a.y - b.y;
        d += dx * dx + dy * dy;
        n += b.x * b.x + b.y * b.y;
    }
    s_d[threadIdx.x] = d;
    s_n[threadIdx.x] = n;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            s_d[threadIdx.x] += s_d[threadIdx.x + o];
            s_n[threadIdx.x] += s_n[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = sqrt(s_d[0]) / sqrt(s_n[0]);
}

// y = C (U (R x)); err = ||y_old - y|| / ||y||. Buffers on the device.
int matvec_err(LegacyCtx &c, const double2 *C, const double2 *U, const double2 *R,
               const double2 *x, const double2 *y_old, double2 *y, double2 *t1, double2 *t2,
               double *d_err, int m, int r, int n) {
    std::vector<ZgemmJob> j1{zjob(R, r, ZOP_N, x, n, ZOP_N, t1, r, r, 1, n)};
    PSKEL_TRY(launch_zgemm(j1, c.stream, c.scratch));
    std::vector<ZgemmJob> j2{zjob(U, r, ZOP_N, t1, r, ZOP_N, t2, r, r, 1, r)};
    PSKEL_TRY(launch_zgemm(j2, c.stream, c.scratch2));
    std::vector<ZgemmJob> j3{zjob(C, m, ZOP_N, t2, r, ZOP_N, y, m, m, 1, r)};
    PSKEL_TRY(launch_zgemm(j3, c.stream, c.scratch));
    err_kernel<<<1, 256, 0, c.stream>>>(y_old, y, m, d_err);
    PSKEL_LAUNCHED(1);
    return PSKEL_OK;
}

// Pseudo-inverse of a device matrix A (M x N) into P (N x M) through the Jacobi SVD; for
// M < N the SVD runs on A^H. Optional outputs: thin left vectors (M x min), singular values
// sorted descending, and the right vectors as rows of Vt (N x N, rows beyond min zero).
struct PinvOut {
    double2 *P = nullptr;      // N x M pinv (device)
    double2 *Uleft = nullptr;  // M x min (device) or null
    double *S = nullptr;       // min (device) or null
    double2 *Vt = nullptr;     // N x N (device) or null, rows scaled by 1/s if vt_scaled
    int vt_scaled = 0;
    double tau = 0;
    int relative = 0;
    int rank = 0;
};

__global__ void conj_transpose_kernel(const double2 *A, int M, int N, double2 *B) {
    // B (N x M) = A^H
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)M * N) return;
    const int i = (int)(idx % M), j = (int)(idx / M);
    const double2 v = A[idx];
    B[j + (size_t)i * N] = make_double2(v.x, -v.y);
}

// From the one-sided Jacobi result (AV with orthogonal columns, V) of an m x n matrix with
// m >= n: left vectors W[:, r] = AV[:, perm r] / s_r, S[r] = s_{perm r}, right vectors
// Vr[:, r] = V[:, perm r]. Writes outputs in the orientation of the original matrix.
__global__ void svd_outputs_kernel(const double2 *AV, const double2 *V, const double *sigma,
                                   const int *perm, int m, int n, int transposed,
                                   double2 *Uleft, double *S, double2 *Vt, int Mo, int No,
                                   int vt_scaled, double thr) {
    // original matrix Mo x No; non-transposed: Mo = m, No = n; transposed: Mo = n, No = m
    const int mn = n;  // min(Mo, No)
    const long long tot_u = (long long)Mo * mn;
    const long long tot_v = (long long)No * No;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < mn && S) S[idx] = sigma[perm[idx]];
    if (Uleft && idx < tot_u) {
        const int i = (int)(idx % Mo), r = (int)(idx / Mo);
        const int c = perm[r];
        const double s = sigma[c];
        double2 v;
        if (!transposed) {
            const double2 a = AV[i + (size_t)c * m];
            v = s > 0 ? make_double2(a.x / s, a.y / s) : make_double2(0, 0);
        } else {
            // A^H = W S V^H  =>  A = V S W^H: left vectors of A are V
            v = V[i + (size_t)c * n];
        }
        Uleft[i + (size_t)r * Mo] = v;
    }
    if (Vt && idx < tot_v) {
        const int r = (int)(idx % No), j = (int)(idx / No);  // Vt(r, j)
        double2 v = make_double2(0, 0);
        if (r < mn) {
            const int c = perm[r];
            const double s = sigma[c];
            double2 x;
            if (!transposed) {
                const double2 vv = V[j + (size_t)c * n];
                x = make_double2(vv.x, -vv.y);  // conj(V)(j, c)
            } else {
                // right vectors of A are the left vectors W of A^H: W = AV / s, Vt = W^H
                const double2 a = AV[j + (size_t)c * m];
                x = s > 0 ? make_double2(a.x / s, -a.y / s) : make_double2(0, 0);
            }
            if (vt_scaled) {
                const double w = (s >= thr && s > 0) ? 1.0 / s : 0.0;
                x.x *= w;
                x.y *= w;
            }
            v = x;
        }
        Vt[r + (size_t)j * No] = v;
    }
}

int device_pinv(LegacyCtx &c, const double2 *d_A, int M, int N, PinvOut &o, int need_sorted) {
    const bool tr = M < N;
    const int m = tr ? N : M, n = tr ? M : N;
    // workspace: AV (m x n), V (n x n), sigma (n), perm (n), rank (1), job
    const size_t bAV = sizeof(double2) * (size_t)m * n, bV = sizeof(double2) * (size_t)n * n;
    const size_t total = bAV + bV + sizeof(double) * n + sizeof(int) * (n + 1) + sizeof(SvdJob) +
                         sizeof(PinvJob) + 6 * 256;
    PSKEL_TRY(c.work.reserve(total));
    char *p = c.work.as<char>();
    auto take = [&](size_t b) { char *q = p; p += (b + 255) & ~size_t(255); return q; };
    double2 *AV = reinterpret_cast<double2 *>(take(bAV));
    double2 *V = reinterpret_cast<double2 *>(take(bV));
    double *sigma = reinterpret_cast<double *>(take(sizeof(double) * n));
    int *perm = reinterpret_cast<int *>(take(sizeof(int) * n));
    int *rank = reinterpret_cast<int *>(take(sizeof(int)));
    SvdJob *d_job = reinterpret_cast<SvdJob *>(take(sizeof(SvdJob)));
    PinvJob *d_pj = reinterpret_cast<PinvJob *>(take(sizeof(PinvJob)));
    if (!tr) {
        PSKEL_CUDA(cudaMemcpyAsync(AV, d_A, bAV, cudaMemcpyDeviceToDevice, c.stream));
    } else {
        const long long tot = (long long)M * N;
        conj_transpose_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, c.stream>>>(d_A, M, N, AV);
        PSKEL_LAUNCHED(1);
    }
    std::vector<SvdJob> hj(1);
    hj[0] = SvdJob{AV, V, sigma, perm, m, n, 0, 0};
    PSKEL_CUDA(cudaMemcpyAsync(d_job, hj.data(), sizeof(SvdJob), cudaMemcpyHostToDevice, c.stream));
    PSKEL_TRY(batched_svd(d_job, hj, 60, c.stream, c.scratch));
    // P for the (possibly transposed) matrix: pinv(A^H) = pinv(A)^H
    double2 *Pt = o.P;
    if (tr) {
        PSKEL_TRY(c.scratch2.reserve(sizeof(double2) * (size_t)M * N));
        Pt = c.scratch2.as<double2>();  // n x m = M x N, pinv of A^H
    }
    PinvJob pj{AV, V, sigma, Pt, rank, m, n, o.tau, o.relative};
    PSKEL_CUDA(cudaMemcpyAsync(d_pj, &pj, sizeof(PinvJob), cudaMemcpyHostToDevice, c.stream));
    const int tiles = ((n + 31) / 32) * ((m + 31) / 32);
    PSKEL_TRY(batched_pinv(d_pj, 1, tiles, c.stream));
    if (tr) {
        const long long tot = (long long)M * N;
        conj_transpose_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, c.stream>>>(Pt, M, N, o.P);
        PSKEL_LAUNCHED(1);
    }
    if (need_sorted && (o.Uleft || o.S || o.Vt)) {
        double smax_thr = o.tau;
        if (o.relative) {
            // the kernel needs the absolute threshold; compute sigma_max on the host after sync
            std::vector<double> hs(n);
            PSKEL_CUDA(cudaMemcpyAsync(hs.data(), sigma, sizeof(double) * n, cudaMemcpyDeviceToHost, c.stream));
            PSKEL_CUDA(cudaStreamSynchronize(c.stream));
            double mx = 0;
            for (double s : hs) mx = std::max(mx, s);
            smax_thr = o.tau * mx;
        }
        const long long tot = std::max<long long>((long long)M * n, (long long)N * N);
        svd_outputs_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, c.stream>>>(
            AV, V, sigma, perm, m, n, tr ? 1 : 0, o.Uleft, o.S, o.Vt, M, N, o.vt_scaled, smax_thr);
        PSKEL_LAUNCHED(1);
    }
    int st[2] = {0, 0};
    PSKEL_CUDA(cudaMemcpyAsync(st, &d_job->status, 2 * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    PSKEL_CUDA(cudaMemcpyAsync(&o.rank, rank, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    PSKEL_CUDA(cudaStreamSynchronize(c.stream));
    if (st[0] != PSKEL_OK) {
        set_error(PSKEL_ERR_NOCONV, "Jacobi SVD did not converge in %d sweeps", st[1]);
        return PSKEL_ERR_NOCONV;
    }
    return PSKEL_OK;
}

}  // namespace
}  // namespace pskel

extern "C" double cuda_complete_compression(
    pskel_c128 *Ccompressed, pskel_c128 *Ucompressed, pskel_c128 *Rcompressed, int cur_order,
    double *vec_time_cuda, double pinv_tol, pskel_c128 *Avtest_old, pskel_c128 *Avtest_new,
    pskel_c128 *vtest, int *col_samples, int *row_samples, int C_blocks_x, int C_blocks_y,
    int C_threads_x, int C_threads_y, int U_blocks_x, int U_blocks_y, int U_threads_x,
    int U_threads_y, int R_blocks_x, int R_blocks_y, int R_threads_x, int R_threads_y,
    pskel_c128 *Ztotal, int field, double k, double eta, double Rinteg_s, double Ranal_s,
    double Rinteg_f, int cor_solid, int flag, int *r1, int *r2, double *vertex, double *topol,
    double *trian, double *edges, double *un, double *ds, double *ln, double *cent, int N,
    int n_r1, int n_r2, int rows_vertex, int cols_vertex, int rows_topol, int cols_topol,
    int rows_trian, int cols_trian, int rows_edges, int cols_edges, int rows_un, int cols_un,
    int rows_ds, int cols_ds, int n_ln, int rows_cent, int cols_cent, int blocks_x, int blocks_y,
    int threads_x, int threads_y, int limx, int limy) {
    (void)C_blocks_x; (void)C_blocks_y; (void)C_threads_x; (void)C_threads_y; (void)U_blocks_x;
    (void)U_blocks_y; (void)U_threads_x; (void)U_threads_y; (void)R_blocks_x; (void)R_blocks_y;
    (void)R_threads_x; (void)R_threads_y; (void)Ztotal; (void)cor_solid; (void)flag; (void)trian;
    (void)un; (void)ds; (void)rows_trian; (void)cols_trian; (void)rows_un; (void)cols_un;
    (void)rows_ds; (void)cols_ds; (void)blocks_x; (void)blocks_y; (void)threads_x;
    (void)threads_y; (void)limx; (void)limy;
    LegacyCtx *cp = ctx();
    if (!cp) return kNaN;
    LegacyCtx &c = *cp;
    std::lock_guard<std::mutex> lk(c.mu);
    auto run_round = [&](double &err) -> int {
        PSKEL_TRY(check_field(field));
        const int r = cur_order;
        if (r <= 0 || r > n_r1 || r > n_r2 || N != cols_edges || !Ccompressed || !Ucompressed ||
            !Rcompressed || !Avtest_old || !Avtest_new || !vtest || !vec_time_cuda) {
            set_error(PSKEL_ERR_ARG, "cuda_complete_compression: cur_order=%d n_r1=%d n_r2=%d", r,
                      n_r1, n_r2);
            return PSKEL_ERR_ARG;
        }
        PSKEL_TRY(ensure_init(c));
        PSKEL_TRY(prepare_mesh(c, vertex, rows_vertex, cols_vertex, topol, rows_topol,
                               cols_topol, edges, rows_edges, cols_edges, ln, n_ln, cent,
                               rows_cent, cols_cent));
        const double *lists[4] = {reinterpret_cast<double *>(r1), reinterpret_cast<double *>(r2),
                                  reinterpret_cast<double *>(row_samples),
                                  reinterpret_cast<double *>(col_samples)};
        const int lens[4] = {n_r1, n_r2, r, r};
        int *d_ids[4];
        PSKEL_TRY(upload_ids(c, lists, lens, 4, N, d_ids));
        const size_t m = n_r1, n = n_r2;
        const size_t nC = m * r, nU = (size_t)r * r, nR = (size_t)r * n;
        const size_t nelem = nC + 2 * nU + nR + n + 2 * m + 2 * (size_t)r + 8;
        PSKEL_TRY(c.out.reserve(sizeof(double2) * nelem));
        double2 *dC = c.out.as<double2>();
        double2 *dCore = dC + nC;
        double2 *dU = dCore + nU;
        double2 *dR = dU + nU;
        double2 *dx = dR + nR;
        double2 *dyo = dx + n;
        double2 *dyn = dyo + m;
        double2 *t1 = dyn + m;
        double2 *t2 = t1 + r;
        double *derr = reinterpret_cast<double *>(t2 + r);
        PSKEL_CUDA(cudaMemcpyAsync(dx, vtest, sizeof(double2) * n, cudaMemcpyHostToDevice, c.stream));
        PSKEL_CUDA(cudaMemcpyAsync(dyo, Avtest_old, sizeof(double2) * m, cudaMemcpyHostToDevice, c.stream));
        PSKEL_CUDA(cudaEventRecord(c.ev0, c.stream));
        std::vector<FillJob> jobs{
            FillJob{d_ids[0], d_ids[3], dC, (int)m, r, (int)m, 0},
            FillJob{d_ids[2], d_ids[3], dCore, r, r, r, 0},
            FillJob{d_ids[2], d_ids[1], dR, r, (int)n, r, 0}};
        PSKEL_TRY(fill_jobs(c, jobs, k, eta, radii_of(Rinteg_s, Ranal_s, Rinteg_f)));
        PinvOut po;
        po.P = dU;
        po.tau = pinv_tol;
        po.relative = 0;
        PSKEL_TRY(device_pinv(c, dCore, r, r, po, 0));
        PSKEL_TRY(matvec_err(c, dC, dU, dR, dx, dyo, dyn, t1, t2, derr, (int)m, r, (int)n));
        PSKEL_CUDA(cudaEventRecord(c.ev1, c.stream));
        PSKEL_TRY(check_flags(c));
        float ms = 0;
        PSKEL_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
        vec_time_cuda[0] = ms;
        PSKEL_CUDA(cudaMemcpy(&err, derr, sizeof(double), cudaMemcpyDeviceToHost));
        PSKEL_CUDA(cudaMemcpy(Ccompressed, dC, sizeof(double2) * nC, cudaMemcpyDeviceToHost));
        PSKEL_CUDA(cudaMemcpy(Ucompressed, dU, sizeof(double2) * nU, cudaMemcpyDeviceToHost));
        PSKEL_CUDA(cudaMemcpy(Rcompressed, dR, sizeof(double2) * nR, cudaMemcpyDeviceToHost));
        PSKEL_CUDA(cudaMemcpy(Avtest_new, dyn, sizeof(double2) * m, cudaMemcpyDeviceToHost));
        return PSKEL_OK;
    };
    double err = kNaN;
    return run_round(err) == PSKEL_OK ? err : kNaN;
}

extern "C" double compute_error_compression(pskel_c128 *C, pskel_c128 *U, pskel_c128 *R,
                                            pskel_c128 *Avtest_old, pskel_c128 *Avtest_new,
                                            pskel_c128 *vtest, int M1, int N1, int M2) {
    LegacyCtx *cp = ctx();
    if (!cp) return kNaN;
    LegacyCtx &c = *cp;
    std::lock_guard<std::mutex> lk(c.mu);
    double err = kNaN;
    auto run = [&]() -> int {
        if (M1 <= 0 || N1 <= 0 || M2 <= 0 || !C || !U || !R || !Avtest_old || !Avtest_new || !vtest) {
            set_error(PSKEL_ERR_ARG, "compute_error_compression: M1=%d N1=%d M2=%d", M1, N1, M2);
            return PSKEL_ERR_ARG;
        }
        PSKEL_TRY(ensure_init(c));
        const size_t nC = (size_t)M1 * N1, nU = (size_t)N1 * N1, nR = (size_t)N1 * M2;
        PSKEL_TRY(c.out.reserve(sizeof(double2) * (nC + nU + nR + M2 + 2 * (size_t)M1 + 2 * (size_t)N1 + 2)));
        double2 *dC = c.out.as<double2>(), *dU = dC + nC, *dR = dU + nU, *dx = dR + nR;
        double2 *dyo = dx + M2, *dyn = dyo + M1, *t1 = dyn + M1, *t2 = t1 + N1;
        double *derr = reinterpret_cast<double *>(t2 + N1);
        PSKEL_CUDA(cudaMemcpyAsync(dC, C, sizeof(double2) * nC, cudaMemcpyHostToDevice, c.stream));
        PSKEL_CUDA(cudaMemcpyAsync(dU, U, sizeof(double2) * nU, cudaMemcpyHostToDevice, c.stream));
        PSKEL_CUDA(cudaMemcpyAsync(dR, R, sizeof(double2) * nR, cudaMemcpyHostToDevice, c.stream));
        PSKEL_CUDA(cudaMemcpyAsync(dx, vtest, sizeof(double2) * M2, cudaMemcpyHostToDevice, c.stream));
        PSKEL_CUDA(cudaMemcpyAsync(dyo, Avtest_old, sizeof(double2) * M1, cudaMemcpyHostToDevice, c.stream));
        PSKEL_TRY(matvec_err(c, dC, dU, dR, dx, dyo, dyn, t1, t2, derr, M1, N1, M2));
        PSKEL_CUDA(cudaMemcpyAsync(Avtest_new, dyn, sizeof(double2) * M1, cudaMemcpyDeviceToHost, c.stream));
        PSKEL_CUDA(cudaMemcpyAsync(&err, derr, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        PSKEL_CUDA(cudaStreamSynchronize(c.stream));
        return PSKEL_OK;
    };
    return run() == PSKEL_OK ? err : kNaN;
}

// Host-side pinv front end shared by aux_pinv_compression and cuda_pinv/cuda_svd.
static int host_pinv(LegacyCtx &c, const pskel_c128 *A, int M, int N, double tau,
                     pskel_c128 *P, pskel_c128 *Uleft, double *S, pskel_c128 *Vt, int vt_scaled) {
    if (M <= 0 || N <= 0 || !A) {
        set_error(PSKEL_ERR_ARG, "pinv: M=%d N=%d", M, N);
        return PSKEL_ERR_ARG;
    }
    PSKEL_TRY(ensure_init(c));
    const size_t nA = (size_t)M * N, mn = std::min(M, N);
    PSKEL_TRY(c.out.reserve(sizeof(double2) * (2 * nA + (size_t)M * mn + (size_t)N * N) +
                            sizeof(double) * mn + 1024));
    double2 *dA = c.out.as<double2>();
    double2 *dP = dA + nA;
    double2 *dU = dP + nA;
    double2 *dVt = dU + (size_t)M * mn;
    double *dS = reinterpret_cast<double *>(dVt + (size_t)N * N);
    PSKEL_CUDA(cudaMemcpyAsync(dA, A, sizeof(double2) * nA, cudaMemcpyHostToDevice, c.stream));
    PinvOut po;
    po.P = dP;
    po.Uleft = Uleft ? dU : nullptr;
    po.S = S ? dS : nullptr;
    po.Vt = Vt ? dVt : nullptr;
    po.vt_scaled = vt_scaled;
    po.tau = tau;
    po.relative = 0;
    PSKEL_TRY(device_pinv(c, dA, M, N, po, 1));
    if (P) PSKEL_CUDA(cudaMemcpy(P, dP, sizeof(double2) * nA, cudaMemcpyDeviceToHost));
    if (Uleft) PSKEL_CUDA(cudaMemcpy(Uleft, dU, sizeof(double2) * (size_t)M * mn, cudaMemcpyDeviceToHost));
    if (S) PSKEL_CUDA(cudaMemcpy(S, dS, sizeof(double) * mn, cudaMemcpyDeviceToHost));
    if (Vt) PSKEL_CUDA(cudaMemcpy(Vt, dVt, sizeof(double2) * (size_t)N * N, cudaMemcpyDeviceToHost));
    return PSKEL_OK;
}

extern "C" int aux_pinv_compression(pskel_c128 *C, pskel_c128 *U, pskel_c128 *R, pskel_c128 *A,
                                    int64_t *row_samples, int64_t *col_samples, int ns, int M,
                                    int N, double tolerance) {
    LegacyCtx *cp = ctx();
    if (!cp) return 0;
    LegacyCtx &c = *cp;
    std::lock_guard<std::mutex> lk(c.mu);
    if (!C || !U || !R || !A || !row_samples || !col_samples || ns <= 0 || M <= 0 || N <= 0) {
        set_error(PSKEL_ERR_ARG, "aux_pinv_compression: ns=%d M=%d N=%d", ns, M, N);
        return 0;
    }
    for (int i = 0; i < ns; ++i)
        if (row_samples[i] < 1 || row_samples[i] > M || col_samples[i] < 1 || col_samples[i] > N) {
            set_error(PSKEL_ERR_RANGE, "aux_pinv_compression: sample %d out of range", i);
            return 0;
        }
    // C = A(:, J), R = A(I, :) are host gathers in the reference too (cur_external_cuda.cu:519-566)
    std::vector<pskel_c128> core((size_t)ns * ns);
    for (int j = 0; j < ns; ++j) {
        const size_t cj = (size_t)(col_samples[j] - 1);
        for (int i = 0; i < M; ++i) C[i + (size_t)j * M] = A[i + cj * M];
        for (int i = 0; i < ns; ++i) core[i + (size_t)j * ns] = A[(size_t)(row_samples[i] - 1) + cj * M];
    }
    for (int j = 0; j < N; ++j)
        for (int i = 0; i < ns; ++i) R[i + (size_t)j * ns] = A[(size_t)(row_samples[i] - 1) + (size_t)j * M];
    return host_pinv(c, core.data(), ns, ns, tolerance, U, nullptr, nullptr, nullptr, 0) == PSKEL_OK ? 1 : 0;
}

extern "C" int cuda_pinv(pskel_c128 *pinvA, pskel_c128 *U, double *S, pskel_c128 *Vt,
                         pskel_c128 *A, int M, int N, double treshold) {
    LegacyCtx *cp = ctx();
    if (!cp) return 0;
    LegacyCtx &c = *cp;
    std::lock_guard<std::mutex> lk(c.mu);
    return host_pinv(c, A, M, N, treshold, pinvA, U, S, Vt, 1) == PSKEL_OK ? 1 : 0;
}

extern "C" int cuda_svd(pskel_c128 *U, double *S, pskel_c128 *Vt, pskel_c128 *A, int M, int N) {
    LegacyCtx *cp = ctx();
    if (!cp) return 0;
    LegacyCtx &c = *cp;
    std::lock_guard<std::mutex> lk(c.mu);
    return host_pinv(c, A, M, N, 0.0, nullptr, U, S, Vt, 0) == PSKEL_OK ? 1 : 0;
}

extern "C" int cuda_svd2(pskel_c128 *U, double *S, pskel_c128 *Vt, pskel_c128 *A, int M, int N) {
    return cuda_svd(U, S, Vt, A, M, N);
}

namespace pskel {
namespace {
__global__ void filter_kernel(double *v, int n, double thr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = v[i] < thr ? 0.0 : 1.0 / v[i];
}
}  // namespace
}  // namespace pskel

extern "C" int cuda_filter(double *V, double treshold, int N) {
    LegacyCtx *cp = ctx();
    if (!cp) return 0;
    LegacyCtx &c = *cp;
    std::lock_guard<std::mutex> lk(c.mu);
    auto run = [&]() -> int {
        if (!V || N < 0) {
            set_error(PSKEL_ERR_ARG, "cuda_filter: N=%d", N);
            return PSKEL_ERR_ARG;
        }
        if (N == 0) return PSKEL_OK;
        PSKEL_TRY(ensure_init(c));
        PSKEL_TRY(c.out.reserve(sizeof(double) * N));
        PSKEL_CUDA(cudaMemcpyAsync(c.out.ptr, V, sizeof(double) * N, cudaMemcpyHostToDevice, c.stream));
        filter_kernel<<<(N + 255) / 256, 256, 0, c.stream>>>(c.out.as<double>(), N, treshold);
        PSKEL_LAUNCHED(1);
        PSKEL_CUDA(cudaMemcpyAsync(V, c.out.ptr, sizeof(double) * N, cudaMemcpyDeviceToHost, c.stream));
        PSKEL_CUDA(cudaStreamSynchronize(c.stream));
        return PSKEL_OK;
    };
    return run() == PSKEL_OK ? 1 : 0;
}
