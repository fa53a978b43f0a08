// Near-field blocks of the MoM matrix and the plane-wave excitation, for the H-matrix product
// (near blocks dense + far blocks compressed) and its iterative solve.
//
// The reference forms whole matrices from block lists built elsewhere
// (compres_single_block_spheres.jl:1404-1505, rebuild_matrix*) and solves them densely or by
// characteristic basis functions (solve_by_CBF, compres_single_block_spheres.jl:983-1017);
// its excitation is test_fields (compres_single_block_spheres_for_sweep2.jl:60-85). Here the
// near blocks of an octree partition (the group pairs that are not far, diagonal included) are
// filled once with the near-field rule and kept on the device next to the compressed far
// blocks; the product Y = Z_near X + sum_far C U R X runs entirely on the device.
//
// Layout: every near block (t, s) is a dense column-major m_t x n_s complex-FP64 matrix in one
// buffer; a block table gives its group id lists and offset. The product reads each block once
// (one CTA per block, 256 threads over its rows, the block's X rows staged in shared memory) and
// adds into Y with FP64 atomics: HBM-bound, 16 bytes per near entry.
#include <cmath>
#include <vector>

#include "engine_internal.cuh"

namespace pskel {
namespace {

constexpr int kNearMvThreads = 256;
constexpr int kNearMvMaxRhs = 16;

struct NearBlock {
    const int *rows, *cols;
    long long off;  // element offset of the block in the near buffer
    int m, n;
};

// Y(rows, :) += Z_b X(cols, :) for every near block b; one CTA per block.
__global__ void __launch_bounds__(kNearMvThreads)
near_matvec_kernel(const NearBlock *__restrict__ blocks, const double2 *__restrict__ data,
                   const double2 *__restrict__ X, int ldx, double2 *__restrict__ Y, int ldy,
                   int nrhs) {
    extern __shared__ double2 xs[];  // n x nrhs
    const NearBlock b = blocks[blockIdx.x];
    for (int e = threadIdx.x; e < b.n * nrhs; e += kNearMvThreads) {
        const int j = e % b.n, q = e / b.n;
        xs[q * b.n + j] = X[(size_t)b.cols[j] + (size_t)q * ldx];
    }
    __syncthreads();
    const double2 *Z = data + b.off;
    for (int i = threadIdx.x; i < b.m; i += kNearMvThreads) {
        double ar[kNearMvMaxRhs], ai[kNearMvMaxRhs];
#pragma unroll
        for (int q = 0; q < kNearMvMaxRhs; ++q) ar[q] = ai[q] = 0.0;
        for (int j = 0; j < b.n; ++j) {
            const double2 z = Z[(size_t)i + (size_t)j * b.m];
#pragma unroll
            for (int q = 0; q < kNearMvMaxRhs; ++q) {
                if (q < nrhs) {
                    const double2 x = xs[q * b.n + j];
                    ar[q] += z.x * x.x - z.y * x.y;
                    ai[q] += z.x * x.y + z.y * x.x;
                }
            }
        }
        const int row = b.rows[i];
#pragma unroll
        for (int q = 0; q < kNearMvMaxRhs; ++q) {
            if (q < nrhs) {
                double *y = reinterpret_cast<double *>(Y + (size_t)row + (size_t)q * ldy);
                atomicAdd(y, ar[q]);
                atomicAdd(y + 1, ai[q]);
            }
        }
    }
}

// E(m) = (l_m / 2) [ (e . rho+_c) exp(-jk k_i . c+) + (e . rho-_c) exp(-jk k_i . c-) ] with
// rho+_c = c(T+) - v+, rho-_c = v- - c(T-), k_i = -(sin th cos ph, sin th sin ph, cos th),
// e = cos(rot) (-sin ph, cos ph, 0) + sin(rot) (cos th cos ph, cos th sin ph, -sin th), angles in
// radians as test_fields forms them (compres_single_block_spheres_for_sweep2.jl:60-85).
__global__ void plane_wave_kernel(const double *__restrict__ vertex, const double *__restrict__ edges,
                                  const double *__restrict__ ln, const double *__restrict__ cent,
                                  int ne, int nt, int nv, double k, double3 ki, double3 ei,
                                  double2 *__restrict__ E, int *flags) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= ne) return;
    const double tp = edges[4 * (size_t)m], tm = edges[4 * (size_t)m + 1];
    const double vp = edges[4 * (size_t)m + 2], vm = edges[4 * (size_t)m + 3];
    if (!(tp >= 1.0 && tp <= (double)nt && tm >= 1.0 && tm <= (double)nt && vp >= 1.0 &&
          vp <= (double)nv && vm >= 1.0 && vm <= (double)nv)) {
        atomicOr(flags, 4);
        E[m] = make_double2(0.0, 0.0);
        return;
    }
    const double *cp = cent + 3 * ((size_t)tp - 1), *cm = cent + 3 * ((size_t)tm - 1);
    const double *ap = vertex + 3 * ((size_t)vp - 1), *am = vertex + 3 * ((size_t)vm - 1);
    const double ph_p = -k * (ki.x * cp[0] + ki.y * cp[1] + ki.z * cp[2]);
    const double ph_m = -k * (ki.x * cm[0] + ki.y * cm[1] + ki.z * cm[2]);
    const double dp = ei.x * (cp[0] - ap[0]) + ei.y * (cp[1] - ap[1]) + ei.z * (cp[2] - ap[2]);
    const double dm = ei.x * (am[0] - cm[0]) + ei.y * (am[1] - cm[1]) + ei.z * (am[2] - cm[2]);
    double sp, cpv, sm, cmv;
    sincos(ph_p, &sp, &cpv);
    sincos(ph_m, &sm, &cmv);
    const double h = 0.5 * ln[m];
    E[m] = make_double2(h * (dp * cpv + dm * cmv), h * (dp * sp + dm * sm));
}

}  // namespace
}  // namespace pskel

using namespace pskel;

extern "C" int pskel_near_build(pskel_ctx *c, const int *nt, const int *ns, int n_near,
                                double rinteg_s, double ranal_s, double rinteg_f, int q_far,
                                long long *bytes) {
    if (!c) {
        set_error(PSKEL_ERR_ARG, "near_build: null context");
        return PSKEL_ERR_ARG;
    }
    PSKEL_CUDA(cudaSetDevice(c->device));
    if (!c->have_mesh || c->n_groups <= 0) {
        set_error(PSKEL_ERR_STATE, "near_build: mesh and groups (pskel_set_blocks) required");
        return PSKEL_ERR_STATE;
    }
    if (n_near < 0 || (n_near > 0 && (!nt || !ns)) || (q_far != 1 && q_far != 7) ||
        !(rinteg_s >= 0) || !(ranal_s >= 0) || !(rinteg_f >= 0)) {
        set_error(PSKEL_ERR_ARG, "near_build: n_near=%d q_far=%d", n_near, q_far);
        return PSKEL_ERR_ARG;
    }
    std::vector<NearBlock> tab(n_near);
    std::vector<FillJob> jobs(n_near);
    long long off = 0;
    const int *gids = c->d_gids.as<int>();
    for (int b = 0; b < n_near; ++b) {
        if (nt[b] < 0 || nt[b] >= c->n_groups || ns[b] < 0 || ns[b] >= c->n_groups) {
            set_error(PSKEL_ERR_ARG, "near_build: group id out of range in pair %d", b);
            return PSKEL_ERR_ARG;
        }
        const int m = c->gptr[nt[b] + 1] - c->gptr[nt[b]], n = c->gptr[ns[b] + 1] - c->gptr[ns[b]];
        tab[b] = NearBlock{gids + c->gptr[nt[b]], gids + c->gptr[ns[b]], off, m, n};
        off += (long long)m * n;
    }
    PSKEL_TRY(c->near_data.reserve(sizeof(double2) * (size_t)(off > 0 ? off : 1)));
    for (int b = 0; b < n_near; ++b)
        jobs[b] = FillJob{tab[b].rows, tab[b].cols, c->near_data.as<double2>() + tab[b].off,
                          tab[b].m, tab[b].n, tab[b].m, 0};
    PSKEL_TRY(c->near_tab.reserve(sizeof(NearBlock) * (size_t)(n_near > 0 ? n_near : 1)));
    if (n_near > 0)
        PSKEL_CUDA(cudaMemcpyAsync(c->near_tab.ptr, tab.data(), sizeof(NearBlock) * n_near,
                                   cudaMemcpyHostToDevice, c->stream));
    NearRadii r;
    r.rinteg_s = rinteg_s;
    r.ranal_s = ranal_s;
    r.rinteg_f = rinteg_f;
    r.q_far = q_far;
    PSKEL_CUDA(cudaMemsetAsync(c->flags.ptr, 0, sizeof(int), c->stream));
    // most near-block entries have every triangle pair outside the radii: fill all with the batched
    // far kernel of the same outside rule, then recompute only the entries with a pair inside a
    // radius or a same-triangle pair with the near kernel
    if (n_near > 0) {
        if (!c->mesh.records(q_far).f64.ptr) PSKEL_TRY(build_records(c->mesh, q_far, c->stream, c->flags.as<int>()));
        int tm, tn;
        fill_tile_shape(PSKEL_C128, q_far, 0, &tm, &tn);
        std::vector<int> prefix(n_near + 1, 0);
        for (int b = 0; b < n_near; ++b)
            prefix[b + 1] = prefix[b] + ((tab[b].m + tm - 1) / tm) * ((tab[b].n + tn - 1) / tn);
        const size_t jb = (sizeof(FillJob) * n_near + 255) & ~size_t(255);
        PSKEL_TRY(c->tmp2.reserve(jb + sizeof(int) * prefix.size() + 256));
        FillJob *d_jobs = c->tmp2.as<FillJob>();
        int *d_prefix = reinterpret_cast<int *>(c->tmp2.as<char>() + jb);
        PSKEL_CUDA(cudaMemcpyAsync(d_jobs, jobs.data(), sizeof(FillJob) * n_near, cudaMemcpyHostToDevice, c->stream));
        PSKEL_CUDA(cudaMemcpyAsync(d_prefix, prefix.data(), sizeof(int) * prefix.size(), cudaMemcpyHostToDevice,
                                   c->stream));
        FillParams fp;
        fp.k = c->em.k;
        fp.eta = c->em.eta;
        fp.r_near = 0;
        fp.q_test = fp.q_src = q_far;
        fp.precision = PSKEL_C128;
        fp.split = 0;
        PSKEL_TRY(launch_fill(c->mesh, fp, d_jobs, d_prefix, n_near, prefix.back(), c->flags.as<int>(), c->stream));
        PSKEL_CUDA(cudaStreamSynchronize(c->stream));  // the host job table goes out of scope below
    }
    PSKEL_TRY(near_fill_jobs(c->mesh, r, c->em.k, c->em.eta, jobs, c->near_jobs, c->near_mom,
                             c->flags.as<int>(), c->stream, true, true));
    int h = 0;
    PSKEL_CUDA(cudaMemcpyAsync(&h, c->flags.ptr, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    PSKEL_CUDA(cudaStreamSynchronize(c->stream));
    if (h & 6) {
        set_error(PSKEL_ERR_RANGE, "near_build: an RWG, triangle or vertex id is out of range");
        return PSKEL_ERR_RANGE;
    }
    int mx = 0;
    for (const NearBlock &b : tab) mx = std::max(mx, b.n);
    c->n_near = n_near;
    c->near_max_n = mx;
    if (bytes) *bytes = off * (long long)sizeof(double2);
    return PSKEL_OK;
}

extern "C" int pskel_near_matvec(pskel_ctx *c, const pskel_c128 *X, int ldx, pskel_c128 *Y,
                                 int ldy, int nrhs, int accumulate, void *stream) {
    if (!c || !X || !Y || nrhs <= 0 || nrhs > kNearMvMaxRhs || ldx < c->mesh.ne ||
        ldy < c->mesh.ne || (accumulate != 0 && accumulate != 1)) {
        set_error(PSKEL_ERR_ARG, "near_matvec: bad arguments (nrhs=%d ldx=%d ldy=%d)", nrhs, ldx, ldy);
        return PSKEL_ERR_ARG;
    }
    if (c->n_near < 0) {
        set_error(PSKEL_ERR_STATE, "near_matvec: no near blocks (pskel_near_build)");
        return PSKEL_ERR_STATE;
    }
    PSKEL_CUDA(cudaSetDevice(c->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);  // NULL: legacy default stream
    if (!accumulate) PSKEL_CUDA(cudaMemsetAsync(Y, 0, sizeof(double2) * (size_t)ldy * nrhs, st));
    if (c->n_near == 0) return PSKEL_OK;
    const size_t smem = sizeof(double2) * (size_t)c->near_max_n * nrhs;
    if (smem > 200 * 1024) {
        set_error(PSKEL_ERR_ARG, "near_matvec: group size x nrhs too large (%d x %d)", c->near_max_n, nrhs);
        return PSKEL_ERR_ARG;
    }
    // the near fill ran on the context's stream
    PSKEL_CUDA(cudaStreamSynchronize(c->stream));
    PSKEL_TRY(ensure_smem_attr(near_matvec_kernel, 200 * 1024));
    near_matvec_kernel<<<c->n_near, kNearMvThreads, smem, st>>>(
        c->near_tab.as<NearBlock>(), c->near_data.as<double2>(),
        reinterpret_cast<const double2 *>(X), ldx, reinterpret_cast<double2 *>(Y), ldy, nrhs);
    PSKEL_LAUNCHED(1);
    return PSKEL_OK;
}

extern "C" int pskel_plane_wave(pskel_ctx *c, double theta_deg, double phi_deg, double rot_deg,
                                pskel_c128 *E, void *stream) {
    if (!c || !E) {
        set_error(PSKEL_ERR_ARG, "plane_wave: null argument");
        return PSKEL_ERR_ARG;
    }
    PSKEL_CUDA(cudaSetDevice(c->device));
    if (!c->have_mesh) {
        set_error(PSKEL_ERR_STATE, "plane_wave: no mesh uploaded");
        return PSKEL_ERR_STATE;
    }
    const double pi = 3.14159265358979323846;
    // as test_fields: th = theta pi / 180, ph = phi / 180 (no pi), rot = rot pi / 180
    const double th = theta_deg * pi / 180.0, ph = phi_deg / 180.0, rot = rot_deg * pi / 180.0;
    const double3 ki = make_double3(-std::sin(th) * std::cos(ph), -std::sin(th) * std::sin(ph), -std::cos(th));
    const double3 ei = make_double3(
        std::cos(rot) * -std::sin(ph) + std::sin(rot) * std::cos(th) * std::cos(ph),
        std::cos(rot) * std::cos(ph) + std::sin(rot) * std::cos(th) * std::sin(ph),
        std::sin(rot) * -std::sin(th));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    PSKEL_CUDA(cudaStreamSynchronize(c->stream));
    const int ne = c->mesh.ne;
    PSKEL_CUDA(cudaMemsetAsync(c->flags.ptr, 0, sizeof(int), st));
    plane_wave_kernel<<<(ne + 255) / 256, 256, 0, st>>>(
        c->mesh.vertex.as<double>(), c->mesh.edges.as<double>(), c->mesh.ln.as<double>(),
        c->mesh.cent.as<double>(), ne, c->mesh.nt, c->mesh.nv, c->em.k, ki, ei,
        reinterpret_cast<double2 *>(E), c->flags.as<int>());
    PSKEL_LAUNCHED(1);
    return PSKEL_OK;
}
