// On-disk format of the compressed far field: the recompressed blocks C' S R' of every far block
// of a partition, with the partition itself, so that a later process can reload them into a
// context and run the tensor-core store matvec without recompressing.
//
// The reference keeps its compressed blocks in Julia/JLD session files (e.g. the
// results_sweep_compression.jld sweeps); it has no store format of its own. Layout
// (little-endian):
//
//   char[8]  magic "PSKELST1"
//   u32      version (1), u32 flags (bit 0: some blocks are transposes of others)
//   i64      N (RWG count), i32 G (groups), i32 B (far blocks), f64 thresh (recompression)
//   i32[G+1] group_ptr, i32[N'] group_ids (N' = group_ptr[G]), i32[B] gt, i32[B] gs
//   i32[4B]  per block: m, n, k, mirror (-1, or the block it is the transpose of)
//   per block with mirror = -1, in block order: C' (m x k complex128, column-major),
//            S (k float64), R' (k x n complex128, column-major)
//   u64      FNV-1a hash of every byte before it
//
// A block with mirror >= 0 stores nothing: its factors are C' = R'_p^T, S = S_p, R' = C'_p^T.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <new>
#include <stdexcept>
#include <vector>

#include "engine_internal.cuh"

namespace pskel {
namespace {

constexpr char kStoreMagic[8] = {'P', 'S', 'K', 'E', 'L', 'S', 'T', '1'};
constexpr unsigned kStoreVersion = 1;

struct Fnv {
    unsigned long long h = 1469598103934665603ull;
    void add(const void *p, size_t n) {
        const unsigned char *b = static_cast<const unsigned char *>(p);
        for (size_t i = 0; i < n; ++i) {
            h ^= b[i];
            h *= 1099511628211ull;
        }
    }
};

struct Writer {
    FILE *f = nullptr;
    Fnv fnv;
    bool ok = true;
    void put(const void *p, size_t n) {
        if (!ok || n == 0) return;
        fnv.add(p, n);
        ok = std::fwrite(p, 1, n, f) == n;
    }
    template <typename T> void put(const T &v) { put(&v, sizeof(T)); }
};

struct Reader {
    FILE *f = nullptr;
    Fnv fnv;
    bool ok = true;
    void get(void *p, size_t n) {
        if (!ok || n == 0) return;
        ok = std::fread(p, 1, n, f) == n;
        if (ok) fnv.add(p, n);
    }
    template <typename T> T get() {
        T v{};
        get(&v, sizeof(T));
        return v;
    }
};

size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace
}  // namespace pskel

using namespace pskel;

extern "C" int pskel_store_save(pskel_ctx *c, const char *path, double thresh) {
    if (!c || !path) {
        set_error(PSKEL_ERR_ARG, "store_save: null argument");
        return PSKEL_ERR_ARG;
    }
    if (c->n_blocks <= 0 || (int)c->recomp_slots.size() != c->n_blocks ||
        (int)c->results.size() != c->n_blocks) {
        set_error(PSKEL_ERR_STATE, "store_save: run pskel_recompress first");
        return PSKEL_ERR_STATE;
    }
    PSKEL_CUDA(cudaSetDevice(c->device));
    PSKEL_CUDA(cudaStreamSynchronize(c->stream));
    Writer w;
    w.f = std::fopen(path, "wb");
    if (!w.f) {
        set_error(PSKEL_ERR_ARG, "store_save: cannot open %s", path);
        return PSKEL_ERR_ARG;
    }
    const int B = c->n_blocks, G = c->n_groups;
    unsigned flags = 0;
    for (int b = 0; b < B; ++b)
        if (c->recomp_slots[b].mirror >= 0) flags |= 1u;
    w.put(kStoreMagic, sizeof(kStoreMagic));
    w.put(kStoreVersion);
    w.put(flags);
    w.put((long long)c->mesh.ne);
    w.put(G);
    w.put(B);
    w.put(thresh);
    w.put(c->gptr.data(), sizeof(int) * c->gptr.size());
    w.put(c->gids.data(), sizeof(int) * c->gids.size());
    w.put(c->gt.data(), sizeof(int) * B);
    w.put(c->gs.data(), sizeof(int) * B);
    for (int b = 0; b < B; ++b) {
        const int rec[4] = {c->results[b].m, c->results[b].n, c->recomp_slots[b].k,
                            c->recomp_slots[b].mirror};
        w.put(rec, sizeof(rec));
    }
    std::vector<double2> hbuf;
    std::vector<double> hs;
    int st = PSKEL_OK;
    for (int b = 0; b < B && w.ok && st == PSKEL_OK; ++b) {
        const RecompSlot &sl = c->recomp_slots[b];
        if (sl.mirror >= 0) continue;
        const BlockResult &res = c->results[b];
        const size_t m = res.m, n = res.n, k = sl.k, ld = sl.ldrp;
        hbuf.resize(std::max(m * k, ld * n) + 1);
        hs.resize(k + 1);
        if (cudaMemcpy(hbuf.data(), sl.Cp, 16 * m * k, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(hs.data(), sl.S, 8 * k, cudaMemcpyDeviceToHost) != cudaSuccess) {
            st = PSKEL_ERR_CUDA;
            break;
        }
        w.put(hbuf.data(), 16 * m * k);
        w.put(hs.data(), 8 * k);
        // R' is kept k x n with leading dimension ldrp >= k: write its first k rows
        if (cudaMemcpy(hbuf.data(), sl.Rp, 16 * ld * n, cudaMemcpyDeviceToHost) != cudaSuccess) {
            st = PSKEL_ERR_CUDA;
            break;
        }
        for (size_t j = 0; j < n; ++j) w.put(hbuf.data() + j * ld, 16 * k);
    }
    if (st == PSKEL_OK && w.ok) {
        const unsigned long long h = w.fnv.h;
        w.put(h);
    }
    const bool closed = std::fclose(w.f) == 0;
    if (st != PSKEL_OK) {
        set_error(st, "store_save: device copy failed");
        return st;
    }
    if (!w.ok || !closed) {
        set_error(PSKEL_ERR_ARG, "store_save: write to %s failed", path);
        return PSKEL_ERR_ARG;
    }
    return PSKEL_OK;
}

static int store_load_impl(pskel_ctx *c, const char *path, int *n_blocks) {
    if (!c || !path) {
        set_error(PSKEL_ERR_ARG, "store_load: null argument");
        return PSKEL_ERR_ARG;
    }
    PSKEL_CUDA(cudaSetDevice(c->device));
    if (!c->have_mesh) {
        set_error(PSKEL_ERR_STATE, "store_load: upload the mesh first");
        return PSKEL_ERR_STATE;
    }
    Reader r;
    r.f = std::fopen(path, "rb");
    if (!r.f) {
        set_error(PSKEL_ERR_ARG, "store_load: cannot open %s", path);
        return PSKEL_ERR_ARG;
    }
    struct Closer {
        FILE *f;
        ~Closer() { std::fclose(f); }
    } closer{r.f};
    // every count read from the header is bounded by the file's size before anything is sized
    // from it, so a corrupt or hostile header cannot ask for more memory than the file holds
    long long fsize = -1;
    if (std::fseek(r.f, 0, SEEK_END) == 0) fsize = std::ftell(r.f);
    if (fsize < 0 || std::fseek(r.f, 0, SEEK_SET) != 0) {
        set_error(PSKEL_ERR_ARG, "store_load: cannot size %s", path);
        return PSKEL_ERR_ARG;
    }
    char magic[8];
    r.get(magic, 8);
    const unsigned version = r.get<unsigned>();
    r.get<unsigned>();  // flags
    const long long N = r.get<long long>();
    const int G = r.get<int>(), B = r.get<int>();
    r.get<double>();  // thresh
    if (!r.ok || std::memcmp(magic, kStoreMagic, 8) != 0 || version != kStoreVersion) {
        set_error(PSKEL_ERR_ARG, "store_load: %s is not a version-%u store file", path, kStoreVersion);
        return PSKEL_ERR_ARG;
    }
    if (N != c->mesh.ne || G <= 0 || B <= 0 || G > (1 << 26) || B > (1 << 28) ||
        4 * ((long long)G + 1) + 24 * (long long)B > fsize) {
        set_error(PSKEL_ERR_ARG, "store_load: N=%lld G=%d B=%d (the mesh has %d RWG)", N, G, B,
                  c->mesh.ne);
        return PSKEL_ERR_ARG;
    }
    std::vector<int> gptr(G + 1), gt(B), gs(B), rec(4 * (size_t)B);
    r.get(gptr.data(), sizeof(int) * gptr.size());
    if (!r.ok || gptr[0] != 0 || gptr[G] <= 0 || gptr[G] > (int)N) {
        set_error(PSKEL_ERR_ARG, "store_load: bad group offsets");
        return PSKEL_ERR_ARG;
    }
    for (int g = 0; g < G; ++g)
        if (gptr[g + 1] < gptr[g]) {
            set_error(PSKEL_ERR_ARG, "store_load: bad group offsets");
            return PSKEL_ERR_ARG;
        }
    if (4 * (long long)gptr[G] > fsize) {
        set_error(PSKEL_ERR_ARG, "store_load: %s is truncated", path);
        return PSKEL_ERR_ARG;
    }
    std::vector<int> gids(gptr[G]);
    r.get(gids.data(), sizeof(int) * gids.size());
    r.get(gt.data(), sizeof(int) * B);
    r.get(gs.data(), sizeof(int) * B);
    r.get(rec.data(), sizeof(int) * rec.size());
    if (!r.ok) {
        set_error(PSKEL_ERR_ARG, "store_load: %s is truncated", path);
        return PSKEL_ERR_ARG;
    }
    // validate the block records against the groups before touching the context
    size_t total = 0;
    for (int b = 0; b < B; ++b) {
        const int m = rec[4 * b], n = rec[4 * b + 1], k = rec[4 * b + 2], mir = rec[4 * b + 3];
        const bool groups_ok = gt[b] >= 0 && gt[b] < G && gs[b] >= 0 && gs[b] < G;
        if (!groups_ok || m != gptr[gt[b] + 1] - gptr[gt[b]] || n != gptr[gs[b] + 1] - gptr[gs[b]] ||
            k < 0 || k > std::min(m, n) || mir >= B ||
            (mir >= 0 && (rec[4 * mir + 3] >= 0 || rec[4 * mir + 2] != k || gt[mir] != gs[b] ||
                          gs[mir] != gt[b]))) {
            set_error(PSKEL_ERR_ARG, "store_load: block record %d is inconsistent", b);
            return PSKEL_ERR_ARG;
        }
        if (mir < 0) total += al256(16 * (size_t)m * k) + al256(8 * (size_t)k) + al256(16 * (size_t)k * n);
    }
    if (total > (size_t)fsize + 256 * (size_t)B * 3) {  // factor bytes plus their padding
        set_error(PSKEL_ERR_ARG, "store_load: %s is truncated", path);
        return PSKEL_ERR_ARG;
    }
    std::vector<char> data(total + 1);
    std::vector<size_t> off(B, 0);
    {
        size_t o = 0;
        for (int b = 0; b < B; ++b) {
            const int m = rec[4 * b], n = rec[4 * b + 1], k = rec[4 * b + 2];
            if (rec[4 * b + 3] >= 0) continue;
            off[b] = o;
            const size_t cm = al256(16 * (size_t)m * k), sk = al256(8 * (size_t)k);
            r.get(data.data() + o, 16 * (size_t)m * k);
            r.get(data.data() + o + cm, 8 * (size_t)k);
            r.get(data.data() + o + cm + sk, 16 * (size_t)k * n);
            o += cm + sk + al256(16 * (size_t)k * n);
        }
    }
    const unsigned long long want = r.fnv.h;
    unsigned long long got = 0;
    if (r.ok && std::fread(&got, sizeof(got), 1, r.f) != 1) r.ok = false;
    if (!r.ok || got != want) {
        set_error(PSKEL_ERR_ARG, "store_load: %s is truncated or corrupt (hash mismatch)", path);
        return PSKEL_ERR_ARG;
    }
    if (std::fgetc(r.f) != EOF) {
        set_error(PSKEL_ERR_ARG, "store_load: %s has bytes after its hash", path);
        return PSKEL_ERR_ARG;
    }
    PSKEL_TRY(pskel_set_blocks(c, gptr.data(), gids.data(), G, gt.data(), gs.data(), B));
    PSKEL_TRY(c->recomp.reserve(total + 256));
    if (total > 0) PSKEL_CUDA(cudaMemcpy(c->recomp.ptr, data.data(), total, cudaMemcpyHostToDevice));
    c->results.assign(B, BlockResult());
    c->recomp_slots.assign(B, RecompSlot{});
    for (int b = 0; b < B; ++b) {
        const int m = rec[4 * b], n = rec[4 * b + 1], k = rec[4 * b + 2], mir = rec[4 * b + 3];
        BlockResult &res = c->results[b];
        res.m = m;
        res.n = n;
        res.r = k;
        res.arena = -1;
        res.mirror = mir;
        if (mir < 0) {
            const size_t cm = al256(16 * (size_t)m * k);
            char *p = c->recomp.as<char>() + off[b];
            RecompSlot &sl = c->recomp_slots[b];
            sl.Cp = reinterpret_cast<double2 *>(p);
            sl.S = reinterpret_cast<double *>(p + cm);
            sl.Rp = reinterpret_cast<double2 *>(p + cm + al256(8 * (size_t)k));
            sl.k = k;
            sl.ldrp = k;  // R' is stored with leading dimension k
            sl.mirror = -1;
        }
    }
    for (int b = 0; b < B; ++b) {
        const int mir = rec[4 * b + 3];
        if (mir >= 0) {
            c->recomp_slots[b] = c->recomp_slots[mir];
            c->recomp_slots[b].mirror = mir;
        }
    }
    ++c->generation;  // the CUR-form tables no longer describe these blocks
    if (n_blocks) *n_blocks = B;
    return PSKEL_OK;
}

extern "C" int pskel_store_load(pskel_ctx *c, const char *path, int *n_blocks) {
    try {
        return store_load_impl(c, path, n_blocks);
    } catch (const std::bad_alloc &) {
        set_error(PSKEL_ERR_OOM, "store_load: out of host memory reading %s", path ? path : "");
        return PSKEL_ERR_OOM;
    } catch (const std::length_error &) {
        set_error(PSKEL_ERR_ARG, "store_load: %s: sizes out of range", path ? path : "");
        return PSKEL_ERR_ARG;
    }
}
