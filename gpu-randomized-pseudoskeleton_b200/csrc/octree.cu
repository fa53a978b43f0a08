// Single-level octree partition of the RWG basis functions and the far-field block list, built
// on the device from the mesh already resident in the context.
//
// The reference has no partitioner of its own: its multi-block driver
// (compres_single_block_spheres.jl:1109-1347) reads block lists produced elsewhere. The partition
// computed here is the one the far-field workloads are defined on, and it reproduces the host
// restatement (pskel/octree.py, partition) bit for bit:
//
//   1. basis centre of RWG e = 0.5 (centroid(T+) + centroid(T-)) (user_get_OG_basis_center.m:36-39);
//   2. origin = 0.5 (min + max) of the centres unless given; box index = floor((c - origin) / leaf);
//   3. Morton key of the box index shifted to start at 0 (21 bits per axis, x lowest);
//   4. stable radix sort of (key, RWG id); groups = runs of equal keys, in key order;
//      group centre = origin + (index of the run's first member + 0.5) leaf;
//   5. groups below min_group folded, smallest first, into the nearest group (size-weighted
//      centre) -- a short sequential loop over the group list, run on the host;
//   6. far pairs (i, j), i != j (i < j when symmetric), with
//      sqrt((dx dx + dy dy) + dz dz) >= admissibility * sqrt(3) * leaf, in row-major order.
//
// Every floating-point step is one IEEE-rounded operation (__dadd_rn & co., no contraction), in
// the order the host restatement evaluates it, so groups, centres and the far list are exact.
// Data layout: centres and box indices are structure-of-arrays (x[N] y[N] z[N]); keys and ids
// are N-long arrays sorted by CUB's onesweep radix sort; the far list is two int arrays.
#include <climits>
#include <cmath>
#include <cstring>
#include <numeric>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_run_length_encode.cuh>
#include <cub/device/device_scan.cuh>

#include "engine_internal.cuh"

using namespace pskel;

namespace {

constexpr int kOctThreads = 256;

struct OctHdr {
    unsigned long long bmin[3], bmax[3];  // order-preserving encodings of the centre bounds
    double origin[3];
    long long imin[3], imax[3];           // box index bounds
    int has_origin;
    int bad;                              // 1: an RWG names a triangle outside the mesh
    int nruns;
    int pad;
};

// Order-preserving map of a double onto unsigned 64-bit integers (for atomic min / max).
__device__ __forceinline__ unsigned long long ord_enc(double x) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(x);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double ord_dec(unsigned long long u) {
    const unsigned long long b = (u >> 63) ? (u & 0x7FFFFFFFFFFFFFFFull) : ~u;
    return __longlong_as_double((long long)b);
}

template <typename T> __device__ __forceinline__ T warp_min(T v) {
    for (int o = 16; o; o >>= 1) {
        const T w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    return v;
}
template <typename T> __device__ __forceinline__ T warp_max(T v) {
    for (int o = 16; o; o >>= 1) {
        const T w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
    }
    return v;
}

// sqrt((dx dx + dy dy) + dz dz), each operation rounded once.
__device__ __forceinline__ double dist3(double ax, double ay, double az, double bx, double by,
                                        double bz) {
    const double dx = __dsub_rn(ax, bx), dy = __dsub_rn(ay, by), dz = __dsub_rn(az, bz);
    return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
}

__global__ void oct_init_kernel(OctHdr *h, int has_origin, double ox, double oy, double oz) {
    if (threadIdx.x != 0) return;
    for (int d = 0; d < 3; ++d) {
        h->bmin[d] = ~0ull;
        h->bmax[d] = 0ull;
        h->imin[d] = LLONG_MAX;
        h->imax[d] = LLONG_MIN;
    }
    h->origin[0] = ox;
    h->origin[1] = oy;
    h->origin[2] = oz;
    h->has_origin = has_origin;
    h->bad = 0;
    h->nruns = 0;
}

// One thread per RWG: its basis centre (SoA) and the running bounds of all centres.
__global__ void __launch_bounds__(kOctThreads)
oct_centre_kernel(const double *__restrict__ edges, const double *__restrict__ cent, int n, int nt,
                  double *__restrict__ c, OctHdr *h) {
    const int e = blockIdx.x * kOctThreads + threadIdx.x;
    unsigned long long lo[3] = {~0ull, ~0ull, ~0ull}, hi[3] = {0ull, 0ull, 0ull};
    if (e < n) {
        const double tpd = edges[4 * (size_t)e], tmd = edges[4 * (size_t)e + 1];
        if (!(tpd >= 1.0 && tpd <= (double)nt && tmd >= 1.0 && tmd <= (double)nt)) {
            atomicOr(&h->bad, 1);
            for (int d = 0; d < 3; ++d) c[(size_t)d * n + e] = 0.0;
        } else {
            const int tp = (int)tpd - 1, tm = (int)tmd - 1;
            for (int d = 0; d < 3; ++d) {
                const double v = __dmul_rn(0.5, __dadd_rn(cent[3 * (size_t)tp + d], cent[3 * (size_t)tm + d]));
                c[(size_t)d * n + e] = v;
                lo[d] = hi[d] = ord_enc(v);
            }
        }
    }
    for (int d = 0; d < 3; ++d) {
        lo[d] = warp_min(lo[d]);
        hi[d] = warp_max(hi[d]);
    }
    if ((threadIdx.x & 31) == 0)
        for (int d = 0; d < 3; ++d) {
            atomicMin(&h->bmin[d], lo[d]);
            atomicMax(&h->bmax[d], hi[d]);
        }
}

// One thread per RWG: box index floor((c - origin) / leaf) per axis and the index bounds.
__global__ void __launch_bounds__(kOctThreads)
oct_box_kernel(const double *__restrict__ c, int n, double leaf, OctHdr *h,
               long long *__restrict__ idx) {
    double o[3];
    const bool given = h->has_origin != 0;
    for (int d = 0; d < 3; ++d)
        o[d] = given ? h->origin[d] : __dmul_rn(0.5, __dadd_rn(ord_dec(h->bmin[d]), ord_dec(h->bmax[d])));
    // the derived origin is kept for the group centres (nothing else reads it in this kernel)
    if (!given && blockIdx.x == 0 && threadIdx.x == 0)
        for (int d = 0; d < 3; ++d) h->origin[d] = o[d];
    const int e = blockIdx.x * kOctThreads + threadIdx.x;
    long long lo[3] = {LLONG_MAX, LLONG_MAX, LLONG_MAX}, hi[3] = {LLONG_MIN, LLONG_MIN, LLONG_MIN};
    if (e < n)
        for (int d = 0; d < 3; ++d) {
            const long long v = (long long)floor(__ddiv_rn(__dsub_rn(c[(size_t)d * n + e], o[d]), leaf));
            idx[(size_t)d * n + e] = v;
            lo[d] = hi[d] = v;
        }
    for (int d = 0; d < 3; ++d) {
        lo[d] = warp_min(lo[d]);
        hi[d] = warp_max(hi[d]);
    }
    if ((threadIdx.x & 31) == 0)
        for (int d = 0; d < 3; ++d) {
            atomicMin(&h->imin[d], lo[d]);
            atomicMax(&h->imax[d], hi[d]);
        }
}

// Spread the low 21 bits of v to every third bit position.
__device__ __forceinline__ unsigned long long spread3(unsigned long long v) {
    v &= 0x1FFFFFull;
    v = (v | (v << 32)) & 0x1F00000000FFFFull;
    v = (v | (v << 16)) & 0x1F0000FF0000FFull;
    v = (v | (v << 8)) & 0x100F00F00F00F00Full;
    v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

__global__ void __launch_bounds__(kOctThreads)
oct_morton_kernel(const long long *__restrict__ idx, int n, const OctHdr *h,
                  unsigned long long *__restrict__ key, int *__restrict__ id) {
    const int e = blockIdx.x * kOctThreads + threadIdx.x;
    if (e >= n) return;
    unsigned long long k = 0;
    for (int d = 0; d < 3; ++d)
        k |= spread3((unsigned long long)(idx[(size_t)d * n + e] - h->imin[d])) << d;
    key[e] = k;
    id[e] = e;
}

// One thread per key run: the box centre of its first member's box, (G, 3) row-major.
__global__ void oct_box_centre_kernel(int g_count, const int *__restrict__ start,
                                      const int *__restrict__ order, const long long *__restrict__ idx,
                                      int n, const OctHdr *h, double leaf, double *__restrict__ bc) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= g_count) return;
    const int first = order[start[g]];
    for (int d = 0; d < 3; ++d) {
        const double o = h->origin[d];
        bc[3 * (size_t)g + d] = __dadd_rn(o, __dmul_rn(__dadd_rn((double)idx[(size_t)d * n + first], 0.5), leaf));
    }
}

// One CTA per key run: final group of each member, scattered to RWG id order.
__global__ void oct_final_key_kernel(const int *__restrict__ start, const int *__restrict__ cnt,
                                     const int *__restrict__ order, const int *__restrict__ map,
                                     unsigned int *__restrict__ fkey) {
    const int g = blockIdx.x;
    const int s = start[g], k = cnt[g];
    const unsigned int f = (unsigned int)map[g];
    for (int i = threadIdx.x; i < k; i += blockDim.x) fkey[order[s + i]] = f;
}

// One CTA per final group: diameter of the bounding sphere about the members' mean centre.
__global__ void __launch_bounds__(kOctThreads)
oct_extent_kernel(const int *__restrict__ gptr, const int *__restrict__ gids,
                  const double *__restrict__ c, int n, double *__restrict__ ext) {
    __shared__ double red[3][kOctThreads / 32];
    __shared__ double mean[3];
    const int g = blockIdx.x, b = gptr[g], k = gptr[g + 1] - b;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double s[3] = {0.0, 0.0, 0.0};
    for (int i = threadIdx.x; i < k; i += kOctThreads) {
        const int e = gids[b + i];
        for (int d = 0; d < 3; ++d) s[d] = __dadd_rn(s[d], c[(size_t)d * n + e]);
    }
    for (int d = 0; d < 3; ++d) {
        for (int o = 16; o; o >>= 1) s[d] = __dadd_rn(s[d], __shfl_xor_sync(0xffffffffu, s[d], o));
        if (lane == 0) red[d][w] = s[d];
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double t = 0.0;
        for (int q = 0; q < kOctThreads / 32; ++q) t = __dadd_rn(t, red[threadIdx.x][q]);
        mean[threadIdx.x] = __ddiv_rn(t, (double)k);
    }
    __syncthreads();
    double m = 0.0;
    for (int i = threadIdx.x; i < k; i += kOctThreads) {
        const int e = gids[b + i];
        const double r = dist3(c[e], c[(size_t)n + e], c[2 * (size_t)n + e], mean[0], mean[1], mean[2]);
        m = r > m ? r : m;
    }
    m = warp_max(m);
    __syncthreads();
    if (lane == 0) red[0][w] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < kOctThreads / 32; ++q) t = red[0][q] > t ? red[0][q] : t;
        ext[g] = __dmul_rn(2.0, t);
    }
}

__device__ __forceinline__ bool oct_far(const double *__restrict__ fc, int i, int j, int g_count,
                                        double ci0, double ci1, double ci2, double thr, int sym) {
    if (j >= g_count || j == i || (sym && j < i)) return false;
    return dist3(ci0, ci1, ci2, fc[3 * (size_t)j], fc[3 * (size_t)j + 1], fc[3 * (size_t)j + 2]) >= thr;
}

// One CTA per group i: the number of far partners j.
__global__ void __launch_bounds__(kOctThreads)
oct_far_count_kernel(const double *__restrict__ fc, int g_count, double thr, int sym,
                     long long *__restrict__ rowcnt) {
    const int i = blockIdx.x;
    const double c0 = fc[3 * (size_t)i], c1 = fc[3 * (size_t)i + 1], c2 = fc[3 * (size_t)i + 2];
    long long total = 0;
    const int j0 = sym ? ((i + 1) / kOctThreads) * kOctThreads : 0;
    for (int jb = j0; jb < g_count; jb += kOctThreads)
        total += __syncthreads_count(oct_far(fc, i, jb + threadIdx.x, g_count, c0, c1, c2, thr, sym));
    if (threadIdx.x == 0) rowcnt[i] = total;
}

// One CTA per group i: its far partners, in ascending j, at rowoff[i].
__global__ void __launch_bounds__(kOctThreads)
oct_far_write_kernel(const double *__restrict__ fc, int g_count, double thr, int sym,
                     const long long *__restrict__ rowoff, int *__restrict__ gt,
                     int *__restrict__ gs) {
    __shared__ int wcount[kOctThreads / 32];
    const int i = blockIdx.x;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const double c0 = fc[3 * (size_t)i], c1 = fc[3 * (size_t)i + 1], c2 = fc[3 * (size_t)i + 2];
    long long base = rowoff[i];
    const int j0 = sym ? ((i + 1) / kOctThreads) * kOctThreads : 0;
    for (int jb = j0; jb < g_count; jb += kOctThreads) {
        const int j = jb + threadIdx.x;
        const bool f = oct_far(fc, i, j, g_count, c0, c1, c2, thr, sym);
        const unsigned bal = __ballot_sync(0xffffffffu, f);
        if (lane == 0) wcount[w] = __popc(bal);
        __syncthreads();
        int off = 0, tot = 0;
        for (int q = 0; q < kOctThreads / 32; ++q) {
            off += q < w ? wcount[q] : 0;
            tot += wcount[q];
        }
        if (f) {
            const long long p = base + off + __popc(bal & ((1u << lane) - 1u));
            gt[p] = i;
            gs[p] = j;
        }
        base += tot;
        __syncthreads();
    }
}

int bit_length(unsigned long long v) {
    int b = 0;
    while (v) {
        ++b;
        v >>= 1;
    }
    return b;
}

// Greedy merge of the groups below min_group, in the host restatement's order: repeatedly the
// smallest group (first of equal sizes) goes into the nearest other group (first of equal
// distances), whose centre becomes the size-weighted mean. Outputs the final group of every
// initial group, the final sizes and centres.
void merge_small_groups(const std::vector<int> &cnt, const std::vector<double> &bc, int min_group,
                        std::vector<int> &map, std::vector<int> &fsize, std::vector<double> &fcen) {
    const int g_count = (int)cnt.size();
    std::vector<long long> size(cnt.begin(), cnt.end());
    std::vector<double> cen(bc);
    std::vector<int> owner(g_count, -1), alive(g_count);
    std::iota(alive.begin(), alive.end(), 0);
    if (min_group > 1 && g_count > 1) {
        while (alive.size() > 1) {
            size_t k = 0;
            for (size_t q = 1; q < alive.size(); ++q)
                if (size[alive[q]] < size[alive[k]]) k = q;
            if (size[alive[k]] >= min_group) break;
            const int i = alive[k];
            int jb = -1;
            double db = 0.0;
            for (int j : alive) {
                if (j == i) continue;
                const double dx = cen[3 * j] - cen[3 * i];
                const double dy = cen[3 * j + 1] - cen[3 * i + 1];
                const double dz = cen[3 * j + 2] - cen[3 * i + 2];
                const double xx = dx * dx, yy = dy * dy, zz = dz * dz;
                const double s2 = xx + yy;
                const double d = std::sqrt(s2 + zz);
                if (jb < 0 || d < db) {
                    jb = j;
                    db = d;
                }
            }
            const double ni = (double)size[i], nj = (double)size[jb], nt = (double)(size[i] + size[jb]);
            for (int d = 0; d < 3; ++d) {
                const double a = cen[3 * jb + d] * nj, b = cen[3 * i + d] * ni;
                const double s = a + b;
                cen[3 * jb + d] = s / nt;
            }
            size[jb] += size[i];
            owner[i] = jb;
            alive.erase(alive.begin() + (long)k);
        }
    }
    std::vector<int> final_of(g_count, -1);
    for (size_t f = 0; f < alive.size(); ++f) final_of[alive[f]] = (int)f;
    map.assign(g_count, 0);
    for (int g = 0; g < g_count; ++g) {
        int r = g;
        while (owner[r] >= 0) r = owner[r];
        map[g] = final_of[r];
    }
    fsize.resize(alive.size());
    fcen.resize(3 * alive.size());
    for (size_t f = 0; f < alive.size(); ++f) {
        fsize[f] = (int)size[alive[f]];
        for (int d = 0; d < 3; ++d) fcen[3 * f + d] = cen[3 * alive[f] + d];
    }
}

int grid_of(long long n) { return (int)((n + kOctThreads - 1) / kOctThreads); }

}  // namespace

namespace pskel {
void octree_release(OctreeState &o) {
    for (DevBuf *b : {&o.hdr, &o.c, &o.idx, &o.ka, &o.kb, &o.va, &o.vb, &o.cnt, &o.start, &o.bc,
                      &o.map, &o.fkey, &o.fkey2, &o.gids, &o.gptr, &o.fc, &o.ext, &o.rowcnt,
                      &o.rowoff, &o.gt, &o.gs, &o.tmp})
        b->release();
    o.valid = false;
}
}  // namespace pskel

extern "C" int pskel_octree_build(pskel_ctx *c, double leaf, const double *origin,
                                  double admissibility, int min_group, int symmetric,
                                  int *n_groups, long long *n_blocks) {
    if (!c) {
        set_error(PSKEL_ERR_ARG, "octree_build: null context");
        return PSKEL_ERR_ARG;
    }
    PSKEL_CUDA(cudaSetDevice(c->device));
    if (!c->have_mesh) {
        set_error(PSKEL_ERR_STATE, "octree_build: no mesh uploaded");
        return PSKEL_ERR_STATE;
    }
    if (!(leaf > 0.0) || !std::isfinite(leaf) || !(admissibility >= 0.0) ||
        !std::isfinite(admissibility) || (symmetric != 0 && symmetric != 1) ||
        (origin && !(std::isfinite(origin[0]) && std::isfinite(origin[1]) && std::isfinite(origin[2])))) {
        set_error(PSKEL_ERR_ARG, "octree_build: leaf > 0, admissibility >= 0, finite origin, symmetric 0/1");
        return PSKEL_ERR_ARG;
    }
    OctreeState &o = c->octree;
    o.valid = false;
    const int n = c->mesh.ne;
    cudaStream_t st = c->stream;
    PSKEL_TRY(o.hdr.reserve(sizeof(OctHdr)));
    PSKEL_TRY(o.c.reserve(sizeof(double) * 3 * (size_t)n));
    PSKEL_TRY(o.idx.reserve(sizeof(long long) * 3 * (size_t)n));
    PSKEL_TRY(o.ka.reserve(sizeof(unsigned long long) * (size_t)n));
    PSKEL_TRY(o.kb.reserve(sizeof(unsigned long long) * (size_t)n));
    PSKEL_TRY(o.va.reserve(sizeof(int) * (size_t)n));
    PSKEL_TRY(o.vb.reserve(sizeof(int) * (size_t)n));
    PSKEL_TRY(o.cnt.reserve(sizeof(int) * (size_t)n));
    PSKEL_TRY(o.start.reserve(sizeof(int) * (size_t)n));
    PSKEL_TRY(o.gids.reserve(sizeof(int) * (size_t)n));
    OctHdr *h = o.hdr.as<OctHdr>();

    oct_init_kernel<<<1, 32, 0, st>>>(h, origin ? 1 : 0, origin ? origin[0] : 0.0,
                                      origin ? origin[1] : 0.0, origin ? origin[2] : 0.0);
    PSKEL_LAUNCHED(1);
    oct_centre_kernel<<<grid_of(n), kOctThreads, 0, st>>>(c->mesh.edges.as<double>(),
                                                           c->mesh.cent.as<double>(), n, c->mesh.nt,
                                                           o.c.as<double>(), h);
    PSKEL_LAUNCHED(1);
    oct_box_kernel<<<grid_of(n), kOctThreads, 0, st>>>(o.c.as<double>(), n, leaf, h,
                                                        o.idx.as<long long>());
    PSKEL_LAUNCHED(1);
    OctHdr hh;
    PSKEL_CUDA(cudaMemcpyAsync(&hh, h, sizeof(OctHdr), cudaMemcpyDeviceToHost, st));
    PSKEL_CUDA(cudaStreamSynchronize(st));
    if (hh.bad) {
        set_error(PSKEL_ERR_RANGE, "octree_build: an RWG names a triangle outside the mesh");
        return PSKEL_ERR_RANGE;
    }
    int bits = 0;
    for (int d = 0; d < 3; ++d) {
        const int b = bit_length((unsigned long long)(hh.imax[d] - hh.imin[d]));
        bits = b > bits ? b : bits;
    }
    bits = bits > 21 ? 21 : bits;
    const int end_bit = bits > 0 ? 3 * bits : 1;
    oct_morton_kernel<<<grid_of(n), kOctThreads, 0, st>>>(o.idx.as<long long>(), n, h,
                                                           o.ka.as<unsigned long long>(), o.va.as<int>());
    PSKEL_LAUNCHED(1);

    // CUB scratch: the largest of the calls below
    size_t tb = 0, t1 = 0;
    PSKEL_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t1, o.ka.as<unsigned long long>(),
                                               o.kb.as<unsigned long long>(), o.va.as<int>(),
                                               o.vb.as<int>(), n, 0, end_bit, st));
    tb = t1 > tb ? t1 : tb;
    PSKEL_CUDA(cub::DeviceRunLengthEncode::Encode(nullptr, t1, o.kb.as<unsigned long long>(),
                                                  o.ka.as<unsigned long long>(), o.cnt.as<int>(),
                                                  &h->nruns, n, st));
    tb = t1 > tb ? t1 : tb;
    PSKEL_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, t1, o.cnt.as<int>(), o.start.as<int>(), n, st));
    tb = t1 > tb ? t1 : tb;
    PSKEL_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t1, o.gids.as<unsigned int>(),
                                               o.gids.as<unsigned int>(), o.va.as<int>(),
                                               o.vb.as<int>(), n, 0, 32, st));
    tb = t1 > tb ? t1 : tb;
    PSKEL_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, t1, o.start.as<long long>(),
                                             o.start.as<long long>(), n + 1, st));
    tb = t1 > tb ? t1 : tb;
    PSKEL_TRY(o.tmp.reserve(tb));

    size_t tsz = o.tmp.bytes;
    PSKEL_CUDA(cub::DeviceRadixSort::SortPairs(o.tmp.ptr, tsz, o.ka.as<unsigned long long>(),
                                               o.kb.as<unsigned long long>(), o.va.as<int>(),
                                               o.vb.as<int>(), n, 0, end_bit, st));
    tsz = o.tmp.bytes;
    PSKEL_CUDA(cub::DeviceRunLengthEncode::Encode(o.tmp.ptr, tsz, o.kb.as<unsigned long long>(),
                                                  o.ka.as<unsigned long long>(), o.cnt.as<int>(),
                                                  &h->nruns, n, st));
    int g0 = 0;
    PSKEL_CUDA(cudaMemcpyAsync(&g0, &h->nruns, sizeof(int), cudaMemcpyDeviceToHost, st));
    PSKEL_CUDA(cudaStreamSynchronize(st));
    if (g0 < 1 || g0 > n) {
        set_error(PSKEL_ERR_CUDA, "octree_build: run count %d outside [1, %d]", g0, n);
        return PSKEL_ERR_CUDA;
    }
    tsz = o.tmp.bytes;
    PSKEL_CUDA(cub::DeviceScan::ExclusiveSum(o.tmp.ptr, tsz, o.cnt.as<int>(), o.start.as<int>(), g0, st));
    PSKEL_TRY(o.bc.reserve(sizeof(double) * 3 * (size_t)g0));
    oct_box_centre_kernel<<<(g0 + 127) / 128, 128, 0, st>>>(g0, o.start.as<int>(), o.vb.as<int>(),
                                                             o.idx.as<long long>(), n, h, leaf,
                                                             o.bc.as<double>());
    PSKEL_LAUNCHED(1);
    std::vector<int> cnt(g0);
    std::vector<double> bc(3 * (size_t)g0);
    PSKEL_CUDA(cudaMemcpyAsync(cnt.data(), o.cnt.ptr, sizeof(int) * g0, cudaMemcpyDeviceToHost, st));
    PSKEL_CUDA(cudaMemcpyAsync(bc.data(), o.bc.ptr, sizeof(double) * 3 * g0, cudaMemcpyDeviceToHost, st));
    PSKEL_CUDA(cudaStreamSynchronize(st));

    std::vector<int> map, fsize;
    merge_small_groups(cnt, bc, min_group, map, fsize, o.h_centres);
    const int gf = (int)fsize.size();
    o.h_gptr.assign(gf + 1, 0);
    for (int f = 0; f < gf; ++f) o.h_gptr[f + 1] = o.h_gptr[f] + fsize[f];
    if (gf == g0) {
        // no merge: the key-sorted ids are the groups (ascending ids within each run)
        PSKEL_CUDA(cudaMemcpyAsync(o.gids.ptr, o.vb.ptr, sizeof(int) * (size_t)n,
                                   cudaMemcpyDeviceToDevice, st));
    } else {
        PSKEL_TRY(o.map.reserve(sizeof(int) * (size_t)g0));
        PSKEL_TRY(o.fkey.reserve(sizeof(unsigned int) * (size_t)n));
        PSKEL_TRY(o.fkey2.reserve(sizeof(unsigned int) * (size_t)n));
        PSKEL_CUDA(cudaMemcpyAsync(o.map.ptr, map.data(), sizeof(int) * g0, cudaMemcpyHostToDevice, st));
        oct_final_key_kernel<<<g0, 128, 0, st>>>(o.start.as<int>(), o.cnt.as<int>(), o.vb.as<int>(),
                                                 o.map.as<int>(), o.fkey.as<unsigned int>());
        PSKEL_LAUNCHED(1);
        // stable sort of the ids 0..N-1 (still in va) by final group: ascending ids per group
        const int fbits = bit_length((unsigned long long)(gf - 1));
        tsz = o.tmp.bytes;
        PSKEL_CUDA(cub::DeviceRadixSort::SortPairs(o.tmp.ptr, tsz, o.fkey.as<unsigned int>(),
                                                   o.fkey2.as<unsigned int>(), o.va.as<int>(),
                                                   o.gids.as<int>(), n, 0, fbits > 0 ? fbits : 1, st));
    }
    PSKEL_TRY(o.gptr.reserve(sizeof(int) * (size_t)(gf + 1)));
    PSKEL_TRY(o.fc.reserve(sizeof(double) * 3 * (size_t)gf));
    PSKEL_TRY(o.ext.reserve(sizeof(double) * (size_t)gf));
    PSKEL_TRY(o.rowcnt.reserve(sizeof(long long) * (size_t)(gf + 1)));
    PSKEL_TRY(o.rowoff.reserve(sizeof(long long) * (size_t)(gf + 1)));
    PSKEL_CUDA(cudaMemcpyAsync(o.gptr.ptr, o.h_gptr.data(), sizeof(int) * (gf + 1), cudaMemcpyHostToDevice, st));
    PSKEL_CUDA(cudaMemcpyAsync(o.fc.ptr, o.h_centres.data(), sizeof(double) * 3 * gf, cudaMemcpyHostToDevice, st));
    oct_extent_kernel<<<gf, kOctThreads, 0, st>>>(o.gptr.as<int>(), o.gids.as<int>(), o.c.as<double>(),
                                                  n, o.ext.as<double>());
    PSKEL_LAUNCHED(1);
    const double diam = std::sqrt(3.0) * leaf;
    const double thr = admissibility * diam;
    PSKEL_CUDA(cudaMemsetAsync(o.rowcnt.ptr, 0, sizeof(long long) * (size_t)(gf + 1), st));
    oct_far_count_kernel<<<gf, kOctThreads, 0, st>>>(o.fc.as<double>(), gf, thr, symmetric,
                                                     o.rowcnt.as<long long>());
    PSKEL_LAUNCHED(1);
    tsz = o.tmp.bytes;
    PSKEL_CUDA(cub::DeviceScan::ExclusiveSum(o.tmp.ptr, tsz, o.rowcnt.as<long long>(),
                                             o.rowoff.as<long long>(), gf + 1, st));
    long long nb = 0;
    PSKEL_CUDA(cudaMemcpyAsync(&nb, o.rowoff.as<long long>() + gf, sizeof(long long),
                               cudaMemcpyDeviceToHost, st));
    PSKEL_CUDA(cudaStreamSynchronize(st));
    if (nb < 0 || nb > (long long)gf * gf || nb > 0x7fffffffLL) {
        set_error(PSKEL_ERR_RANGE, "octree_build: %lld far pairs (limit 2^31 - 1)", nb);
        return PSKEL_ERR_RANGE;
    }
    PSKEL_TRY(o.gt.reserve(sizeof(int) * (size_t)(nb > 0 ? nb : 1)));
    PSKEL_TRY(o.gs.reserve(sizeof(int) * (size_t)(nb > 0 ? nb : 1)));
    if (nb > 0) {
        oct_far_write_kernel<<<gf, kOctThreads, 0, st>>>(o.fc.as<double>(), gf, thr, symmetric,
                                                         o.rowoff.as<long long>(), o.gt.as<int>(),
                                                         o.gs.as<int>());
        PSKEL_LAUNCHED(1);
    }
    PSKEL_CUDA(cudaStreamSynchronize(st));
    o.n = n;
    o.n_groups = gf;
    o.n_blocks = nb;
    o.valid = true;
    if (n_groups) *n_groups = gf;
    if (n_blocks) *n_blocks = nb;
    return PSKEL_OK;
}

extern "C" int pskel_octree_get(pskel_ctx *c, int *group_ptr, int *group_ids, double *centres,
                                double *extents, int *gt, int *gs) {
    if (!c) {
        set_error(PSKEL_ERR_ARG, "octree_get: null context");
        return PSKEL_ERR_ARG;
    }
    PSKEL_CUDA(cudaSetDevice(c->device));
    const OctreeState &o = c->octree;
    if (!o.valid) {
        set_error(PSKEL_ERR_STATE, "octree_get: no octree built");
        return PSKEL_ERR_STATE;
    }
    cudaStream_t st = c->stream;
    if (group_ptr) std::memcpy(group_ptr, o.h_gptr.data(), sizeof(int) * (o.n_groups + 1));
    if (centres) std::memcpy(centres, o.h_centres.data(), sizeof(double) * 3 * o.n_groups);
    if (group_ids)
        PSKEL_CUDA(cudaMemcpyAsync(group_ids, o.gids.ptr, sizeof(int) * (size_t)o.n, cudaMemcpyDeviceToHost, st));
    if (extents)
        PSKEL_CUDA(cudaMemcpyAsync(extents, o.ext.ptr, sizeof(double) * (size_t)o.n_groups, cudaMemcpyDeviceToHost, st));
    if (gt && o.n_blocks > 0)
        PSKEL_CUDA(cudaMemcpyAsync(gt, o.gt.ptr, sizeof(int) * (size_t)o.n_blocks, cudaMemcpyDeviceToHost, st));
    if (gs && o.n_blocks > 0)
        PSKEL_CUDA(cudaMemcpyAsync(gs, o.gs.ptr, sizeof(int) * (size_t)o.n_blocks, cudaMemcpyDeviceToHost, st));
    PSKEL_CUDA(cudaStreamSynchronize(st));
    return PSKEL_OK;
}
