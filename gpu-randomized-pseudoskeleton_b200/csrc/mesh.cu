// Mesh upload, per-RWG quadrature records and id conversion.
#include <atomic>
#include <cstdarg>
#include <cmath>

#include "pskel_internal.cuh"

namespace pskel {

// ------------------------------------------------------------------ thread-local errors
static thread_local int g_code = PSKEL_OK;
static thread_local char g_msg[512] = "ok";

void set_error(int code, const char *fmt, ...) {
    g_code = code;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_msg, sizeof(g_msg), fmt, ap);
    va_end(ap);
}
int last_code() { return g_code; }

static std::atomic<long long> g_launches{0};
void count_launch(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
long long launches_so_far() { return g_launches.load(std::memory_order_relaxed); }

int sm_count() {
    static std::atomic<int> counts[kMaxDevices];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= kMaxDevices) dev = 0;
    int n = counts[dev].load(std::memory_order_relaxed);
    if (n <= 0) {
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
        counts[dev].store(n, std::memory_order_relaxed);
    }
    return n;
}

static SmemAttrTable g_smem_attrs;

int ensure_smem_attr(const void *func, size_t bytes) {
    int dev = 0;
    PSKEL_CUDA(cudaGetDevice(&dev));
    cudaError_t err = cudaSuccess;
    const bool ok = g_smem_attrs.raise(func, dev, bytes, [&](size_t b) {
        err = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b);
        return err == cudaSuccess;
    });
    if (!ok) {
        set_error(PSKEL_ERR_CUDA, "cudaFuncSetAttribute(%zu bytes of shared memory) on device %d: %s",
                  bytes, dev, cudaGetErrorString(err));
        return PSKEL_ERR_CUDA;
    }
    return PSKEL_OK;
}

// ------------------------------------------------------------------ 7-point rule
// Radon's 7-point degree-5 rule (Dunavant 1985, n = 5): centroid weight 9/40; points
// (a, a, 1-2a) with a = (6 -+ sqrt 15)/21 and weights (155 -+ sqrt 15)/1200 (weights sum to 1).
struct Rule7 {
    double a[7], b[7], c[7], w[7];
};
static Rule7 make_rule7() {
    Rule7 r;
    const double s15 = std::sqrt(15.0);
    const double A[2] = {(6.0 - s15) / 21.0, (6.0 + s15) / 21.0};
    const double W[2] = {(155.0 - s15) / 1200.0, (155.0 + s15) / 1200.0};
    r.a[0] = r.b[0] = r.c[0] = 1.0 / 3.0;
    r.w[0] = 9.0 / 40.0;
    int k = 1;
    for (int g = 0; g < 2; ++g) {
        const double a = A[g], b = 1.0 - 2.0 * a;
        const double bc[3][3] = {{b, a, a}, {a, b, a}, {a, a, b}};
        for (int p = 0; p < 3; ++p, ++k) {
            r.a[k] = bc[p][0];
            r.b[k] = bc[p][1];
            r.c[k] = bc[p][2];
            r.w[k] = W[g];
        }
    }
    return r;
}

void quadrature_weights(int q, double *w) {
    if (q == 1) {
        w[0] = 1.0;
        return;
    }
    static const Rule7 r7 = make_rule7();
    for (int i = 0; i < 7; ++i) w[i] = r7.w[i];
}

struct RuleArg {
    double a[7], b[7], c[7], w[7];
};

// One thread per (RWG e, side, point p): writes the 7 fields of that point.
__global__ void build_records_kernel(const double *__restrict__ vertex,
                                     const double *__restrict__ topol,
                                     const double *__restrict__ edges,
                                     const double *__restrict__ ln,
                                     const double *__restrict__ cent, int ne, int nt, int nv,
                                     int q, RuleArg rule, double *__restrict__ rec64, int *flags) {
    const int np = 2 * q;
    const int stride = (7 * np) | 1;
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= (long long)ne * np) return;
    const int e = (int)(gid / np);
    const int pp = (int)(gid % np);
    const int side = pp / q;
    const int p = pp % q;
    const int t = (int)edges[4 * (size_t)e + side] - 1;
    const int vo = (int)edges[4 * (size_t)e + 2 + side] - 1;
    double x[3] = {0, 0, 0}, rho[3] = {0, 0, 0};
    double w = 1.0;
    const double s = side == 0 ? 1.0 : -1.0;
    const double l = ln[e];
    bool ok = t >= 0 && t < nt && vo >= 0 && vo < nv;
    if (ok) {
        if (q == 1) {
            for (int d = 0; d < 3; ++d) x[d] = cent[3 * (size_t)t + d];
        } else {
            const int v1 = (int)topol[3 * (size_t)t + 0] - 1;
            const int v2 = (int)topol[3 * (size_t)t + 1] - 1;
            const int v3 = (int)topol[3 * (size_t)t + 2] - 1;
            ok = v1 >= 0 && v1 < nv && v2 >= 0 && v2 < nv && v3 >= 0 && v3 < nv;
            if (ok) {
                for (int d = 0; d < 3; ++d)
                    x[d] = rule.a[p] * vertex[3 * (size_t)v1 + d] +
                           rule.b[p] * vertex[3 * (size_t)v2 + d] +
                           rule.c[p] * vertex[3 * (size_t)v3 + d];
            }
            w = rule.w[p];
        }
        if (ok)
            for (int d = 0; d < 3; ++d) rho[d] = s * (x[d] - vertex[3 * (size_t)vo + d]);
    }
    if (!ok) atomicOr(flags, 2);
    double f[7];
    f[0] = x[0];
    f[1] = x[1];
    f[2] = x[2];
    f[3] = w * 0.5 * l * rho[0];
    f[4] = w * 0.5 * l * rho[1];
    f[5] = w * 0.5 * l * rho[2];
    f[6] = w * s * l;
    double *r64 = rec64 + (size_t)e * stride;
    for (int k = 0; k < 7; ++k) r64[k * np + pp] = f[k];
    if (pp == 0) r64[stride - 1] = 0.0;
}

// One thread per triangle: its q quadrature points and centroid (q = 1 uses the stored centroid
// as its point, like the per-RWG records).
__global__ void build_tri_records_kernel(const double *__restrict__ vertex,
                                         const double *__restrict__ topol,
                                         const double *__restrict__ cent, int nt, int nv, int q,
                                         RuleArg rule, double *__restrict__ out, int *flags) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    double *o = out + (size_t)t * tri_stride(q);
    const int v1 = (int)topol[3 * (size_t)t + 0] - 1;
    const int v2 = (int)topol[3 * (size_t)t + 1] - 1;
    const int v3 = (int)topol[3 * (size_t)t + 2] - 1;
    const bool ok = v1 >= 0 && v1 < nv && v2 >= 0 && v2 < nv && v3 >= 0 && v3 < nv;
    if (!ok) atomicOr(flags, 2);
    for (int p = 0; p < q; ++p)
        for (int d = 0; d < 3; ++d) {
            double x = 0.0;
            if (q == 1) x = cent[3 * (size_t)t + d];
            else if (ok)
                x = rule.a[p] * vertex[3 * (size_t)v1 + d] + rule.b[p] * vertex[3 * (size_t)v2 + d] +
                    rule.c[p] * vertex[3 * (size_t)v3 + d];
            o[3 * p + d] = x;
        }
    for (int d = 0; d < 3; ++d) o[3 * q + d] = cent[3 * (size_t)t + d];
}

int upload_mesh_arrays(DevMesh &mesh, const double *vertex, int nv, const double *topol, int nt,
                       const double *edges, int ne, const double *ln, const double *cent,
                       cudaStream_t stream) {
    if (!vertex || !topol || !edges || !ln || !cent || nv <= 0 || nt <= 0 || ne <= 0) {
        set_error(PSKEL_ERR_ARG, "mesh: null array or empty mesh");
        return PSKEL_ERR_ARG;
    }
    PSKEL_TRY(mesh.vertex.reserve(sizeof(double) * 3 * (size_t)nv));
    PSKEL_TRY(mesh.topol.reserve(sizeof(double) * 3 * (size_t)nt));
    PSKEL_TRY(mesh.edges.reserve(sizeof(double) * 4 * (size_t)ne));
    PSKEL_TRY(mesh.ln.reserve(sizeof(double) * (size_t)ne));
    PSKEL_TRY(mesh.cent.reserve(sizeof(double) * 3 * (size_t)nt));
    PSKEL_CUDA(cudaMemcpyAsync(mesh.vertex.ptr, vertex, sizeof(double) * 3 * (size_t)nv,
                               cudaMemcpyHostToDevice, stream));
    PSKEL_CUDA(cudaMemcpyAsync(mesh.topol.ptr, topol, sizeof(double) * 3 * (size_t)nt,
                               cudaMemcpyHostToDevice, stream));
    PSKEL_CUDA(cudaMemcpyAsync(mesh.edges.ptr, edges, sizeof(double) * 4 * (size_t)ne,
                               cudaMemcpyHostToDevice, stream));
    PSKEL_CUDA(cudaMemcpyAsync(mesh.ln.ptr, ln, sizeof(double) * (size_t)ne,
                               cudaMemcpyHostToDevice, stream));
    PSKEL_CUDA(cudaMemcpyAsync(mesh.cent.ptr, cent, sizeof(double) * 3 * (size_t)nt,
                               cudaMemcpyHostToDevice, stream));
    mesh.nv = nv;
    mesh.nt = nt;
    mesh.ne = ne;
    mesh.rec1.q = 0;  // records are stale until rebuilt
    mesh.rec7.q = 0;
    return PSKEL_OK;
}

int build_records(DevMesh &mesh, int q, cudaStream_t stream, int *d_flag) {
    if (q != 1 && q != 7) {
        set_error(PSKEL_ERR_ARG, "quadrature order must be 1 or 7 (got %d)", q);
        return PSKEL_ERR_ARG;
    }
    MeshRecords &rec = mesh.records(q);
    const size_t n = (size_t)mesh.ne * rec_stride(q);
    PSKEL_TRY(rec.f64.reserve(n * sizeof(double)));
    static const Rule7 r7 = make_rule7();
    RuleArg ra;
    for (int i = 0; i < 7; ++i) {
        ra.a[i] = r7.a[i];
        ra.b[i] = r7.b[i];
        ra.c[i] = r7.c[i];
        ra.w[i] = r7.w[i];
    }
    const long long total = (long long)mesh.ne * rec_points(q);
    const int threads = 256;
    const int blocks = (int)((total + threads - 1) / threads);
    build_records_kernel<<<blocks, threads, 0, stream>>>(
        mesh.vertex.as<double>(), mesh.topol.as<double>(), mesh.edges.as<double>(),
        mesh.ln.as<double>(), mesh.cent.as<double>(), mesh.ne, mesh.nt, mesh.nv, q, ra,
        rec.f64.as<double>(), d_flag);
    PSKEL_LAUNCHED(1);
    PSKEL_TRY(rec.tri.reserve(sizeof(double) * (size_t)mesh.nt * tri_stride(q)));
    build_tri_records_kernel<<<(mesh.nt + 255) / 256, 256, 0, stream>>>(
        mesh.vertex.as<double>(), mesh.topol.as<double>(), mesh.cent.as<double>(), mesh.nt,
        mesh.nv, q, ra, rec.tri.as<double>(), d_flag);
    PSKEL_LAUNCHED(1);
    rec.q = q;
    return PSKEL_OK;
}

// ------------------------------------------------------------------ id conversion
__global__ void ids_from_double_kernel(const double *__restrict__ in, int *__restrict__ out, int n,
                                       int limit, int *flags) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = in[i];
    int id = (int)v - 1;
    if (!(v >= 1.0 && v <= (double)limit) || (double)(id + 1) != v) {
        atomicOr(flags, 4);
        id = 0;
    }
    out[i] = id;
}

__global__ void ids_from_int64_kernel(const long long *__restrict__ in, int *__restrict__ out,
                                      int n, int limit, int *flags) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long v = in[i];
    int id = (int)(v - 1);
    if (v < 1 || v > limit) {
        atomicOr(flags, 4);
        id = 0;
    }
    out[i] = id;
}

int launch_ids_from_double(const double *d_in, int *d_out, int n, int limit, int *d_flags,
                           cudaStream_t stream) {
    if (n <= 0) return PSKEL_OK;
    ids_from_double_kernel<<<(n + 255) / 256, 256, 0, stream>>>(d_in, d_out, n, limit, d_flags);
    PSKEL_LAUNCHED(1);
    return PSKEL_OK;
}

int launch_ids_from_int64(const int64_t *d_in, int *d_out, int n, int limit, int *d_flags,
                          cudaStream_t stream) {
    if (n <= 0) return PSKEL_OK;
    ids_from_int64_kernel<<<(n + 255) / 256, 256, 0, stream>>>(
        reinterpret_cast<const long long *>(d_in), d_out, n, limit, d_flags);
    PSKEL_LAUNCHED(1);
    return PSKEL_OK;
}

}  // namespace pskel

extern "C" int pskel_last_error(const char **message) {
    if (message) *message = pskel::g_msg;
    return pskel::g_code;
}
