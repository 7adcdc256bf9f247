// ft_capi.cu -- the extern "C" boundary (include/fasttree_b200.h): argument checks, host
// pointer staging, tree allocation and error mapping around the build and query kernels.
#include <cuda_runtime.h>

#include <climits>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "ft_common.cuh"
#include "ft_internal.h"

namespace ft {

static thread_local std::string g_last_error;

void fail(ft_status s, const std::string &msg) { throw Error{s, msg}; }

void check_cuda(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return;
    cudaGetLastError();
    ft_status s = (e == cudaErrorMemoryAllocation) ? FT_ERR_OUT_OF_MEMORY : FT_ERR_CUDA;
    fail(s, std::string(what) + ": " + cudaGetErrorString(e));
}

// Makes ctx->device current for the duration of a call and restores the caller's device.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        FT_CUDA(cudaGetDevice(&prev));
        if (prev != dev) FT_CUDA(cudaSetDevice(dev));
    }
    ~DeviceGuard() {
        int cur = -1;
        if (cudaGetDevice(&cur) == cudaSuccess && prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

// Host pointer check: the reference stages exactly the pointers that are not USM
// allocations (sycl::usm::alloc::unknown, src/hlbvh.hpp:131-137); here, pointers the CUDA
// runtime does not know (pageable host memory).
static bool is_host_only(const void *p) {
    if (!p) return false;
    cudaPointerAttributes a;
    cudaError_t           e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return true;
    }
    return a.type == cudaMemoryTypeUnregistered;
}

// Host memory of either kind (pinned or pageable): not device memory or managed memory.
static bool is_host_memory(const void *p) {
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return true;
    }
    return a.type == cudaMemoryTypeUnregistered || a.type == cudaMemoryTypeHost;
}

// Stream-ordered staging of one host buffer (ensure_device_readable / _writable and
// copy_back_and_free, src/hlbvh.hpp:125-200).
struct Staged {
    void        *host  = nullptr;
    void        *dev   = nullptr;
    size_t       bytes = 0;
    bool         owned = false;
    bool         out   = false;
    cudaStream_t st    = nullptr;
    Staged()           = default;
    Staged(const Staged &) = delete;
    Staged &operator=(const Staged &) = delete;
    void init(const void *p, size_t nbytes, bool readable, bool writable, cudaStream_t s) {
        host  = const_cast<void *>(p);
        bytes = nbytes;
        st    = s;
        out   = writable;
        if (!p || nbytes == 0 || !is_host_only(p)) {
            dev = host;
            return;
        }
        FT_CUDA(cudaMallocAsync(&dev, nbytes, st));
        owned = true;
        if (readable) FT_CUDA(cudaMemcpyAsync(dev, p, nbytes, cudaMemcpyHostToDevice, st));
    }
    void copy_back() {
        if (owned && out) FT_CUDA(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, st));
    }
    ~Staged() {
        if (owned) cudaFreeAsync(dev, st);
    }
};

static void validate_options(const ft_options &o) {
    if (o.coord_type < F32 || o.coord_type > U64) fail(FT_ERR_INVALID_ARGUMENT, "unknown coord_type");
    if (o.sfc_type != MORTON && o.sfc_type != PEANO_HILBERT) fail(FT_ERR_INVALID_ARGUMENT, "unknown sfc_type");
    if (o.sfc_type == MORTON && (o.coord_type == U32 || o.coord_type == U64))
        fail(FT_ERR_INVALID_ARGUMENT, "Morton keys are defined for floating-point coordinates only");
}

void check_device_status(uint32_t *status, cudaStream_t st) {
    uint32_t v = 0;
    FT_CUDA(cudaMemcpyAsync(&v, status, sizeof(v), cudaMemcpyDeviceToHost, st));
    FT_CUDA(cudaStreamSynchronize(st));
    if (!v) return;
    FT_CUDA(cudaMemsetAsync(status, 0, sizeof(uint32_t), st));
    FT_CUDA(cudaStreamSynchronize(st));
    if (v & STATUS_BAD_INPUT)
        fail(FT_ERR_INVALID_ARGUMENT, "bad input on the device: a leaf id outside [0, num_leaves), or batch set "
                                      "offsets that do not start at 0, end at num_points and increase");
    if (v & STATUS_SPIN_LIMIT) fail(FT_ERR_TIMEOUT, "a bounded device-side wait gave up (radix-sort look-back)");
    fail(FT_ERR_RUNTIME, "a traversal exceeded its visit bound (corrupt tree)");
}

static void check_status_word(TreeImpl &s, cudaStream_t st) { check_device_status(s.status, st); }

// ---------------------------------------------------------------------------------------
// Tree storage
// ---------------------------------------------------------------------------------------
static void tree_free_arrays(ft_tree &t) {
    void *ptrs[] = {t.min_x, t.max_x, t.min_y, t.max_y, t.min_z, t.max_z, t.left_child,
                    t.right_child, t.parent, t.id, t.is_ghost, t.orig_idx};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    t.min_x = t.max_x = t.min_y = t.max_y = t.min_z = t.max_z = nullptr;
    t.left_child = t.right_child = t.parent = nullptr;
    t.id                                    = nullptr;
    t.is_ghost                              = nullptr;
    t.orig_idx                              = nullptr;
    t.capacity                              = 0;
}

static void *tree_alloc(size_t bytes, bool managed) {
    void *p = nullptr;
    if (bytes == 0) return nullptr;
    cudaError_t e = managed ? cudaMallocManaged(&p, bytes) : cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        fail(FT_ERR_OUT_OF_MEMORY, "tree allocation failed");
    }
    return p;
}

static void tree_alloc_arrays(Context &ctx, ft_tree &t, size_t cap) {
    bool   m   = ctx.opts.host_readable_tree != 0;
    size_t tot = cap > 0 ? 2 * cap - 1 : 0;
    size_t ni  = cap > 0 ? cap - 1 : 0;
    size_t cb  = coord_bytes(ctx.opts.coord_type);
    try {
        t.min_x       = tree_alloc(tot * cb, m);
        t.max_x       = tree_alloc(tot * cb, m);
        t.min_y       = tree_alloc(tot * cb, m);
        t.max_y       = tree_alloc(tot * cb, m);
        t.min_z       = tree_alloc(tot * cb, m);
        t.max_z       = tree_alloc(tot * cb, m);
        t.left_child  = (int32_t *)tree_alloc(ni * 4, m);
        t.right_child = (int32_t *)tree_alloc(ni * 4, m);
        t.parent      = (int32_t *)tree_alloc(tot * 4, m);
        t.id          = (uint32_t *)tree_alloc(tot * 4, m);
        t.is_ghost    = (int8_t *)tree_alloc(tot, m);
        t.orig_idx    = (int32_t *)tree_alloc(tot * 4, m);
    } catch (...) {
        tree_free_arrays(t);
        throw;
    }
    t.capacity = cap;
}

} // namespace ft

using namespace ft;

struct ft_context : public ft::Context {};

#define FT_API_BEGIN try {
#define FT_API_END                                                                                \
    }                                                                                             \
    catch (const ft::Error &e) {                                                                  \
        ft::g_last_error = e.msg;                                                                 \
        return e.status;                                                                          \
    }                                                                                             \
    catch (const std::bad_alloc &) {                                                              \
        ft::g_last_error = "host allocation failed";                                              \
        return FT_ERR_OUT_OF_MEMORY;                                                              \
    }                                                                                             \
    catch (...) {                                                                                 \
        ft::g_last_error = "unknown error";                                                       \
        return FT_ERR_RUNTIME;                                                                    \
    }                                                                                             \
    return FT_OK;

static void need(bool c, const char *msg) {
    if (!c) fail(FT_ERR_INVALID_ARGUMENT, msg);
}
static void need(bool c, const std::string &msg) {
    if (!c) fail(FT_ERR_INVALID_ARGUMENT, msg);
}

// Trees handed out by ft_batch_tree live inside their batch.
static void need_owned(const ft_tree *t) {
    if (t && t->impl && ((const TreeImpl *)t->impl)->view)
        fail(FT_ERR_INVALID_ARGUMENT, "a set view of a batch cannot be rebuilt, resized or destroyed");
}

// Arguments of the batched entry points must be device-accessible (no staging: the calls
// are asynchronous and may be captured in a CUDA graph).
static void need_device(const void *p, const char *what) {
    if (p && is_host_only(p)) fail(FT_ERR_INVALID_ARGUMENT, std::string(what) + " must be device memory");
}

struct ft_batch {
    ft::BatchImpl *impl;
};

struct ft_bound_model {
    ft::BoundModel *impl;
};

extern "C" {

const char *ft_last_error(void) { return ft::g_last_error.c_str(); }

int ft_version(void) { return 10000; }

ft_status ft_context_create(const ft_options *opts, int device, ft_context **out) {
    FT_API_BEGIN
    need(opts && out, "null argument");
    validate_options(*opts);
    int count = 0;
    FT_CUDA(cudaGetDeviceCount(&count));
    need(device >= 0 && device < count, "device ordinal out of range");
    DeviceGuard g(device);
    ft_context *c = new ft_context();
    c->opts       = *opts;
    c->device     = device;
    if (cudaMalloc(&c->status, 32) != cudaSuccess || cudaMemset(c->status, 0, 32) != cudaSuccess) {
        cudaGetLastError();
        delete c;
        fail(FT_ERR_CUDA, "device status word allocation failed");
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) c->num_sms = prop.multiProcessorCount;
    else cudaGetLastError();
    *out = c;
    FT_API_END
}

ft_status ft_context_destroy(ft_context *ctx) {
    if (ctx) {
        if (ctx->status) cudaFree(ctx->status);
        if (ctx->replay_ranks) cudaFree(ctx->replay_ranks);
        if (ctx->replay_rows) cudaFree(ctx->replay_rows);
        if (ctx->seed_ranks) cudaFree(ctx->seed_ranks);
        if (ctx->miss_ranks) cudaFree(ctx->miss_ranks);
        if (ctx->miss_rows) cudaFree(ctx->miss_rows);
        for (int b = 0; b < 2; ++b) {
            if (ctx->stage_idx[b]) cudaFree(ctx->stage_idx[b]);
            if (ctx->stage_dist[b]) cudaFree(ctx->stage_dist[b]);
            if (ctx->ev_walked[b]) cudaEventDestroy(ctx->ev_walked[b]);
            if (ctx->ev_copied[b]) cudaEventDestroy(ctx->ev_copied[b]);
        }
        if (ctx->iota) cudaFree(ctx->iota);
        if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
        ft::free_query_sort(*ctx);
        for (int i = 0; i < ft::BS_COUNT; ++i)
            if (ctx->bprof.ev[i]) cudaEventDestroy(ctx->bprof.ev[i]);
        if (ctx->learned_feats) cudaFree(ctx->learned_feats);
        if (ctx->learned_bound) cudaFree(ctx->learned_bound);
    }
    delete ctx;
    return FT_OK;
}

ft_status ft_check_device_status(ft_context *ctx, ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx != nullptr, "null context");
    DeviceGuard g(ctx->device);
    check_device_status(ctx->status, (cudaStream_t)stream);
    FT_API_END
}

ft_status ft_get_query_stats(ft_context *ctx, ft_query_stats *out) {
    FT_API_BEGIN
    need(ctx && out, "null argument");
    if (ctx->last_fast) { // replay count of the last fast self-kNN (synchronises the device)
        DeviceGuard g(ctx->device);
        uint32_t    w[7] = {0, 0, 0, 0, 0, 0, 0};
        FT_CUDA(cudaMemcpy(w, ctx->status + 1, sizeof(w), cudaMemcpyDeviceToHost));
        ctx->stats.replayed = w[0];
        unsigned long long v, v2;
        std::memcpy(&v, &w[1], sizeof(v));
        std::memcpy(&v2, &w[5], sizeof(v2));
        ctx->stats.reserved[0] = (int64_t)(v + v2); // lane-node visits of the fast walk (both launches)
        ctx->stats.reserved[1] = (int64_t)w[3];     // bound misses rerun by the walk without the bound
        ctx->stats.reserved[2] = (int64_t)v2;       // visits of that rerun
    }
    *out = ctx->stats;
    FT_API_END
}

ft_status ft_get_replayed_queries(ft_context *ctx, int32_t *rows_out, size_t capacity, size_t *count_out) {
    FT_API_BEGIN
    need(ctx && count_out, "null argument");
    need(rows_out || capacity == 0, "null rows_out");
    *count_out = 0;
    if (!ctx->last_fast || !ctx->last_rows || !ctx->replay_rows) return FT_OK;
    DeviceGuard g(ctx->device);
    uint32_t    cnt = 0;
    FT_CUDA(cudaDeviceSynchronize());
    FT_CUDA(cudaMemcpy(&cnt, ctx->status + 1, sizeof(cnt), cudaMemcpyDeviceToHost));
    const size_t c = std::min<size_t>(cnt, ctx->replay_cap);
    *count_out     = c;
    if (capacity > 0 && c > 0)
        FT_CUDA(cudaMemcpy(rows_out, ctx->replay_rows, std::min(c, capacity) * sizeof(int32_t),
                           cudaMemcpyDeviceToHost));
    FT_API_END
}

ft_status ft_tree_create(ft_context *ctx, size_t n, ft_tree **out) {
    FT_API_BEGIN
    need(ctx && out, "null argument");
    DeviceGuard g(ctx->device);
    ft_tree *t = new ft_tree();
    std::memset(t, 0, sizeof(*t));
    TreeImpl *impl = new TreeImpl();
    impl->coord    = ctx->opts.coord_type;
    t->impl        = impl;
    try {
        tree_alloc_arrays(*ctx, *t, n);
    } catch (...) {
        delete impl;
        delete t;
        throw;
    }
    t->num_leaves   = n;
    t->num_internal = n > 0 ? n - 1 : 0;
    *out            = t;
    FT_API_END
}

ft_status ft_tree_ensure(ft_context *ctx, ft_tree *t, size_t n) {
    FT_API_BEGIN
    need(ctx && t, "null argument");
    need_owned(t);
    DeviceGuard g(ctx->device);
    if (n > t->capacity) { // TreePool::ensure (src/hlbvh.hpp:691-705)
        tree_free_arrays(*t);
        tree_alloc_arrays(*ctx, *t, n + n / 2 + 1024);
    }
    t->num_leaves   = n;
    t->num_internal = n > 0 ? n - 1 : 0;
    FT_API_END
}

ft_status ft_tree_destroy(ft_context *ctx, ft_tree *t) {
    FT_API_BEGIN
    if (!t) return FT_OK;
    need(ctx != nullptr, "null context");
    need_owned(t);
    DeviceGuard g(ctx->device);
    tree_free_arrays(*t);
    if (t->impl) {
        TreeImpl *impl = (TreeImpl *)t->impl;
        free_scratch(*impl);
        delete impl;
    }
    delete t;
    FT_API_END
}

ft_status ft_tree_height(ft_context *ctx, const ft_tree *t, int *height_out) {
    FT_API_BEGIN
    need(ctx && t && height_out, "null argument");
    *height_out = ((TreeImpl *)t->impl)->height_root;
    FT_API_END
}

ft_status ft_compute_bbox(ft_context *ctx, const void *x, const void *y, const void *z, size_t n, void *out6,
                          ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx && out6, "null argument");
    DeviceGuard  g(ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    size_t       cb = coord_bytes(ctx->opts.coord_type);
    if (n > 0) need(x && y && z, "null coordinate array");
    Staged sx, sy, sz;
    sx.init(x, n * cb, true, false, st);
    sy.init(y, n * cb, true, false, st);
    sz.init(z, n * cb, true, false, st);
    TreeImpl tmp;
    void    *out_dev = nullptr;
    FT_CUDA(cudaMallocAsync(&tmp.bbox_partial, 1184 * 6 * 8, st));
    FT_CUDA(cudaMallocAsync(&out_dev, 6 * 8, st));
    ft::compute_bbox(*ctx, &tmp, sx.dev, sy.dev, sz.dev, n, out_dev, st);
    FT_CUDA(cudaMemcpyAsync(out6, out_dev, 6 * cb, cudaMemcpyDeviceToHost, st));
    cudaFreeAsync(tmp.bbox_partial, st);
    cudaFreeAsync(out_dev, st);
    tmp.bbox_partial = nullptr;
    FT_CUDA(cudaStreamSynchronize(st));
    FT_API_END
}

ft_status ft_sfc_encode(ft_context *ctx, const void *x, const void *y, const void *z, size_t n, void *keys,
                        const void *bbox6, ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx != nullptr, "null context");
    if (n == 0) return FT_OK;
    need(x && y && z && keys, "null argument");
    bool is_float = ctx->opts.coord_type == F32 || ctx->opts.coord_type == F64;
    need(!is_float || bbox6, "floating-point encoding needs a bounding box");
    DeviceGuard  g(ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    size_t       cb = coord_bytes(ctx->opts.coord_type);
    Staged       sx, sy, sz, sk;
    sx.init(x, n * cb, true, false, st);
    sy.init(y, n * cb, true, false, st);
    sz.init(z, n * cb, true, false, st);
    sk.init(keys, n * ref_key_bytes(ctx->opts), false, true, st);
    TreeImpl tmp;
    void    *bb = nullptr;
    FT_CUDA(cudaMallocAsync((void **)&tmp.key_lo, n * 8, st));
    FT_CUDA(cudaMallocAsync((void **)&tmp.key_hi, n * 8, st));
    FT_CUDA(cudaMallocAsync((void **)&tmp.perm, n * 4, st));
    FT_CUDA(cudaMallocAsync(&bb, 6 * 8, st));
    if (bbox6) FT_CUDA(cudaMemcpyAsync(bb, bbox6, 6 * cb, cudaMemcpyHostToDevice, st));
    else FT_CUDA(cudaMemsetAsync(bb, 0, 6 * 8, st));
    sfc_encode_ref_layout(*ctx, tmp, sx.dev, sy.dev, sz.dev, n, bb, sk.dev, st);
    sk.copy_back();
    cudaFreeAsync(tmp.key_lo, st);
    cudaFreeAsync(tmp.key_hi, st);
    cudaFreeAsync(tmp.perm, st);
    cudaFreeAsync(bb, st);
    tmp.key_lo = tmp.key_hi = nullptr;
    tmp.perm                = nullptr;
    FT_CUDA(cudaStreamSynchronize(st));
    FT_API_END
}

static bool root_in_period(const ft_context *ctx, const ft_tree *tree, cudaStream_t st);

// ---------------------------------------------------------------------------------------
// Tree serialisation (raw SoA arrays + sorted keys behind a fixed header)
// ---------------------------------------------------------------------------------------
struct TreeFileHeader {
    char     magic[8];   // "FTB2TREE"
    uint32_t version;    // 1
    int32_t  coord_type, sfc_type, periodic, key_words, own_keys, clean42_ok, reserved0;
    uint64_t n;
    uint64_t bbox[6];    // build box, each coordinate in an 8-byte slot
    uint8_t  pad[128 - 8 - 4 - 7 * 4 - 8 - 48];
};
static_assert(sizeof(TreeFileHeader) == 128, "tree file header size");

struct TreeSection {
    void  *dev;   // device array of the tree
    size_t bytes; // its size in the file
};

static size_t align16(size_t v) { return (v + 15) & ~size_t(15); }

static std::vector<TreeSection> tree_sections(const ft_context &ctx, const ft_tree &t, size_t n) {
    const TreeImpl &impl = *(const TreeImpl *)t.impl;
    const size_t    cb   = coord_bytes(ctx.opts.coord_type);
    const size_t    nn   = n ? 2 * n - 1 : 0, ni = n ? n - 1 : 0;
    std::vector<TreeSection> v = {{t.min_x, nn * cb},      {t.max_x, nn * cb},       {t.min_y, nn * cb},
                                  {t.max_y, nn * cb},      {t.min_z, nn * cb},       {t.max_z, nn * cb},
                                  {t.left_child, ni * 4},  {t.right_child, ni * 4},  {t.parent, nn * 4},
                                  {t.id, nn * 4},          {t.is_ghost, nn},         {t.orig_idx, nn * 4},
                                  {impl.key_lo, n * 8}};
    if (ctx.opts.coord_type == FT_COORD_U64) v.push_back({impl.key_hi, n * 8});
    return v;
}

static size_t tree_file_bytes(const std::vector<TreeSection> &secs) {
    size_t b = sizeof(TreeFileHeader);
    for (const TreeSection &s : secs) b += align16(s.bytes);
    return b;
}

ft_status ft_tree_export(ft_context *ctx, const ft_tree *tree, void *buf, size_t *bytes, ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx && tree && bytes, "null argument");
    const TreeImpl &impl = *(const TreeImpl *)tree->impl;
    const size_t    n    = tree->num_leaves;
    need(n == 0 || impl.height_root >= 0, "tree export: the tree has not been built");
    need(n == 0 || impl.key_lo, "tree export: the tree has no keys");
    DeviceGuard  g(ctx->device);
    cudaStream_t st   = (cudaStream_t)stream;
    auto         secs = tree_sections(*ctx, *tree, n);
    const size_t need_bytes = tree_file_bytes(secs);
    if (!buf) {
        *bytes = need_bytes;
        return FT_OK;
    }
    need(*bytes >= need_bytes, "tree export: buffer too small (" + std::to_string(*bytes) + " < " +
                                   std::to_string(need_bytes) + " bytes)");
    TreeFileHeader h;
    std::memset(&h, 0, sizeof(h));
    std::memcpy(h.magic, "FTB2TREE", 8);
    h.version    = 1;
    h.coord_type = ctx->opts.coord_type;
    h.sfc_type   = ctx->opts.sfc_type;
    h.periodic   = ctx->opts.periodic;
    h.key_words  = ctx->opts.coord_type == FT_COORD_U64 ? 2 : 1;
    h.own_keys   = impl.own_keys ? 1 : 0;
    h.clean42_ok = impl.clean42_ok ? 1 : 0;
    h.n          = n;
    const size_t cb = coord_bytes(ctx->opts.coord_type);
    if (n && impl.bbox) {
        unsigned char box[48];
        FT_CUDA(cudaMemcpyAsync(box, impl.bbox, 6 * cb, cudaMemcpyDeviceToHost, st));
        FT_CUDA(cudaStreamSynchronize(st));
        for (int i = 0; i < 6; ++i) std::memcpy(&h.bbox[i], box + i * cb, cb);
    }
    unsigned char *out = (unsigned char *)buf;
    FT_CUDA(cudaMemcpyAsync(out, &h, sizeof(h), cudaMemcpyDefault, st));
    size_t off = sizeof(h);
    for (const TreeSection &s : secs) {
        if (s.bytes) FT_CUDA(cudaMemcpyAsync(out + off, s.dev, s.bytes, cudaMemcpyDefault, st));
        const size_t padded = align16(s.bytes);
        static const unsigned char zeros[16] = {}; // padding (buf may be host or device memory)
        if (padded > s.bytes) FT_CUDA(cudaMemcpyAsync(out + off + s.bytes, zeros, padded - s.bytes, cudaMemcpyDefault, st));
        off += padded;
    }
    FT_CUDA(cudaStreamSynchronize(st));
    *bytes = need_bytes;
    FT_API_END
}

ft_status ft_tree_import(ft_context *ctx, const void *buf, size_t bytes, ft_tree *tree, ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx && tree && buf, "null argument");
    need_owned(tree);
    need(bytes >= sizeof(TreeFileHeader), "tree import: buffer smaller than the header");
    DeviceGuard  g(ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    TreeFileHeader h;
    FT_CUDA(cudaMemcpyAsync(&h, buf, sizeof(h), cudaMemcpyDefault, st));
    FT_CUDA(cudaStreamSynchronize(st));
    need(std::memcmp(h.magic, "FTB2TREE", 8) == 0, "tree import: not a fasttree_b200 tree (bad magic)");
    need(h.version == 1, "tree import: unsupported format version " + std::to_string(h.version));
    need(h.coord_type == ctx->opts.coord_type && h.sfc_type == ctx->opts.sfc_type &&
             (h.periodic != 0) == (ctx->opts.periodic != 0),
         "tree import: the context's coordinate type, SFC or periodic option differs from the tree's");
    need(h.n <= (size_t)(INT_MAX / 2), "tree import: leaf count out of range");
    const size_t n = (size_t)h.n;
    need(tree->capacity >= n, "tree import: tree capacity is smaller than the stored leaf count");
    TreeImpl &impl = *(TreeImpl *)tree->impl;
    if (n) ensure_scratch(impl, ctx->opts, n);
    tree->num_leaves   = n;
    tree->num_internal = n ? n - 1 : 0;
    auto secs          = tree_sections(*ctx, *tree, n);
    need(bytes >= tree_file_bytes(secs), "tree import: buffer shorter than the stored arrays");
    const unsigned char *in  = (const unsigned char *)buf;
    size_t               off = sizeof(h);
    for (const TreeSection &s : secs) {
        if (s.bytes) FT_CUDA(cudaMemcpyAsync(s.dev, in + off, s.bytes, cudaMemcpyDefault, st));
        off += align16(s.bytes);
    }
    const size_t cb = coord_bytes(ctx->opts.coord_type);
    unsigned char box[48];
    for (int i = 0; i < 6; ++i) std::memcpy(box + i * cb, &h.bbox[i], cb);
    impl.height_root = -1;
    if (n) {
        FT_CUDA(cudaMemcpyAsync(impl.bbox, box, 6 * cb, cudaMemcpyHostToDevice, st));
        recompute_from_keys(*ctx, *tree, st);
    }
    if (n > 1) {
        uint8_t hr = 0;
        FT_CUDA(cudaMemcpyAsync(&hr, impl.height, 1, cudaMemcpyDeviceToHost, st));
        check_status_word(impl, st);
        impl.height_root = hr;
    } else {
        FT_CUDA(cudaStreamSynchronize(st));
        impl.height_root = 0;
    }
    impl.own_keys   = h.own_keys != 0;
    impl.clean42_ok = h.clean42_ok != 0;
    impl.in_period = root_in_period(ctx, tree, st);
    impl.clean42   = impl.clean42_ok && ctx->opts.coord_type == FT_COORD_U64 && impl.in_period;
    FT_API_END
}

// Root box maxima of an integer tree below the period 2^42 (64-bit) / 2^21 (32-bit), i.e.
// every coordinate is (TreeImpl::in_period).  Blocking.
static bool root_in_period(const ft_context *ctx, const ft_tree *tree, cudaStream_t st) {
    const int ct = ctx->opts.coord_type;
    if (ct == FT_COORD_F32 || ct == FT_COORD_F64 || tree->num_leaves == 0) return true;
    const void *src[3] = {tree->max_x, tree->max_y, tree->max_z};
    if (ct == FT_COORD_U64) {
        uint64_t m[3] = {0, 0, 0};
        for (int a = 0; a < 3; ++a) FT_CUDA(cudaMemcpyAsync(&m[a], src[a], 8, cudaMemcpyDefault, st));
        FT_CUDA(cudaStreamSynchronize(st));
        return m[0] < (1ull << 42) && m[1] < (1ull << 42) && m[2] < (1ull << 42);
    }
    uint32_t m[3] = {0, 0, 0};
    for (int a = 0; a < 3; ++a) FT_CUDA(cudaMemcpyAsync(&m[a], src[a], 4, cudaMemcpyDefault, st));
    FT_CUDA(cudaStreamSynchronize(st));
    return m[0] < (1u << 21) && m[1] < (1u << 21) && m[2] < (1u << 21);
}

ft_status ft_refit_bvh(ft_context *ctx, const void *x, const void *y, const void *z, size_t n, int leaf_order,
                       ft_tree *tree, ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx && tree, "null argument");
    need_owned(tree);
    need(n == tree->num_leaves, "refit: n must equal the tree's leaf count (build the tree first)");
    if (n == 0) return FT_OK;
    need(x && y && z, "null coordinate array");
    TreeImpl &impl = *(TreeImpl *)tree->impl;
    need(impl.height_root >= 0, "refit: the tree has not been built");
    DeviceGuard  g(ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    size_t       cb = coord_bytes(ctx->opts.coord_type);
    Staged       sx, sy, sz;
    sx.init(x, n * cb, true, false, st);
    sy.init(y, n * cb, true, false, st);
    sz.init(z, n * cb, true, false, st);
    ft::refit_bvh(*ctx, *tree, sx.dev, sy.dev, sz.dev, n, leaf_order != 0, st);
    // the 42-bit periodic fast form needs every coordinate below 2^42: the root box's maxima
    uint64_t mx[3] = {0, 0, 0};
    if (ctx->opts.coord_type == FT_COORD_U64) {
        FT_CUDA(cudaMemcpyAsync(&mx[0], tree->max_x, 8, cudaMemcpyDefault, st));
        FT_CUDA(cudaMemcpyAsync(&mx[1], tree->max_y, 8, cudaMemcpyDefault, st));
        FT_CUDA(cudaMemcpyAsync(&mx[2], tree->max_z, 8, cudaMemcpyDefault, st));
    }
    check_status_word(impl, st);
    impl.clean42 = impl.clean42_ok && ctx->opts.coord_type == FT_COORD_U64 && mx[0] < (1ull << 42) &&
                   mx[1] < (1ull << 42) && mx[2] < (1ull << 42);
    impl.in_period = root_in_period(ctx, tree, st);
    FT_API_END
}

ft_status ft_build_bvh(ft_context *ctx, const void *x, const void *y, const void *z, size_t n, const uint32_t *id,
                       const int8_t *is_ghost, const void *bbox6, void *keys, ft_tree *tree, ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx && tree, "null argument");
    need_owned(tree);
    if (n == 0) return FT_OK; // src/hlbvh.hpp:2174
    if (n > (size_t)(INT_MAX / 2))
        fail(FT_ERR_RUNTIME, "Particle count n exceeds maximum supported tree size (INT_MAX / 2).");
    need(x && y && z, "null coordinate array");
    need(tree->capacity >= n, "tree capacity is smaller than the particle count");
    DeviceGuard  g(ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    size_t       cb = coord_bytes(ctx->opts.coord_type);
    Staged       sx, sy, sz, sid, sgh, sk;
    sx.init(x, n * cb, true, false, st);
    sy.init(y, n * cb, true, false, st);
    sz.init(z, n * cb, true, false, st);
    sid.init(id, id ? n * 4 : 0, true, false, st);
    sgh.init(is_ghost, is_ghost ? n : 0, true, false, st);
    sk.init(keys, keys ? n * ref_key_bytes(ctx->opts) : 0, true, true, st);
    tree->num_leaves   = n;
    tree->num_internal = n - 1;
    TreeImpl &impl     = *(TreeImpl *)tree->impl;
    impl.height_root   = -1;
    impl.clean42       = false;
    impl.own_keys      = false;
    ft::build_bvh(*ctx, *tree, sx.dev, sy.dev, sz.dev, n, (const uint32_t *)sid.dev, (const int8_t *)sgh.dev, bbox6,
                  sk.dev, st);
    impl.own_keys = keys == nullptr; // the sorted keys are this library's encoding of bbox
    if (keys) sk.copy_back();
    uint64_t box[6] = {0, 0, 0, 0, 0, 0};
    if (ctx->opts.coord_type == FT_COORD_U64)
        FT_CUDA(cudaMemcpyAsync(box, impl.bbox, sizeof(box), cudaMemcpyDeviceToHost, st));
    if (n > 1) {
        uint8_t h = 0;
        FT_CUDA(cudaMemcpyAsync(&h, impl.height, 1, cudaMemcpyDeviceToHost, st));
        check_status_word(impl, st);
        impl.height_root = h;
    } else {
        check_status_word(impl, st);
        impl.height_root = 0;
    }
    // boxes of a 42-bit tree stay below 2^42 when every coordinate does (max entries 1, 3, 5)
    impl.clean42 = ctx->opts.coord_type == FT_COORD_U64 && box[1] < (1ull << 42) && box[3] < (1ull << 42) &&
                   box[5] < (1ull << 42);
    impl.clean42_ok = true;
    impl.in_period  = root_in_period(ctx, tree, st);
    FT_API_END
}

ft_status ft_build_tree(ft_context *ctx, ft_tree *tree, const void *sorted_keys, const void *sorted_x,
                        const void *sorted_y, const void *sorted_z, const uint32_t *sorted_id,
                        const int8_t *sorted_is_ghost, const int32_t *sorted_orig_idx, ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx && tree, "null argument");
    need_owned(tree);
    size_t n = tree->num_leaves;
    if (n == 0) return FT_OK;
    need(sorted_keys != nullptr, "null key array");
    need(tree->capacity >= n, "tree capacity is smaller than num_leaves");
    DeviceGuard  g(ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    size_t       cb = coord_bytes(ctx->opts.coord_type);
    bool         xyz = sorted_x && sorted_y && sorted_z;
    Staged       sk, sx, sy, sz, sid, sgh, sor;
    sk.init(sorted_keys, n * ref_key_bytes(ctx->opts), true, false, st);
    sx.init(xyz ? sorted_x : nullptr, n * cb, true, false, st);
    sy.init(xyz ? sorted_y : nullptr, n * cb, true, false, st);
    sz.init(xyz ? sorted_z : nullptr, n * cb, true, false, st);
    sid.init(sorted_id, sorted_id ? n * 4 : 0, true, false, st);
    sgh.init(sorted_is_ghost, sorted_is_ghost ? n : 0, true, false, st);
    sor.init(sorted_orig_idx, sorted_orig_idx ? n * 4 : 0, true, false, st);
    tree->num_internal = n - 1;
    TreeImpl &impl     = *(TreeImpl *)tree->impl;
    impl.clean42       = false; // caller leaf arrays: the general periodic distance form
    impl.clean42_ok    = false;
    impl.own_keys      = false;
    impl.height_root   = -1;
    build_tree_from_keys(*ctx, *tree, sk.dev, sx.dev, sy.dev, sz.dev, (const uint32_t *)sid.dev,
                         (const int8_t *)sgh.dev, (const int32_t *)sor.dev, st);
    if (n > 1) {
        uint8_t h = 0;
        FT_CUDA(cudaMemcpyAsync(&h, impl.height, 1, cudaMemcpyDeviceToHost, st));
        check_status_word(impl, st);
        impl.height_root = h;
    } else {
        check_status_word(impl, st);
        impl.height_root = 0;
    }
    impl.in_period = root_in_period(ctx, tree, st);
    FT_API_END
}

ft_status ft_self_knn(ft_context *ctx, const ft_tree *tree, const int32_t *leaf_ids, size_t num, int k,
                      int exclude_self, uint64_t *idx_out, void *dist_out, const ft_query_options *qopts,
                      ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx && tree, "null argument");
    ft_query_options q{};
    if (qopts) q = *qopts;
    if (!leaf_ids) num = tree->num_leaves;
    if (num > 0 && k > 0 && tree->num_leaves > 0) need(idx_out && dist_out, "null output array");
    DeviceGuard g(ctx->device);
    const bool host_idx = is_host_memory(idx_out), host_dist = is_host_memory(dist_out);
    need(host_idx == host_dist, "idx_out and dist_out must both be host or both be device memory");
    if (host_idx) // results straight to host memory, copy-out overlapped with the walk
        ft::self_knn_to_host(*ctx, *tree, leaf_ids, num, k, exclude_self != 0, idx_out, dist_out, q,
                             (cudaStream_t)stream);
    else
        ft::self_knn(*ctx, *tree, leaf_ids, num, k, exclude_self != 0, idx_out, dist_out, q, (cudaStream_t)stream);
    FT_API_END
}

ft_status ft_self_knn_bounded(ft_context *ctx, const ft_tree *tree, const int32_t *leaf_ids, size_t num, int k,
                              int exclude_self, const void *bound, uint64_t *idx_out, void *dist_out,
                              const ft_query_options *qopts, ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx && tree, "null argument");
    ft_query_options q{};
    if (qopts) q = *qopts;
    if (!leaf_ids) num = tree->num_leaves;
    if (num > 0 && k > 0 && tree->num_leaves > 0) need(idx_out && dist_out && bound, "null array argument");
    need_device(bound, "bound");
    DeviceGuard g(ctx->device);
    ft::self_knn(*ctx, *tree, leaf_ids, num, k, exclude_self != 0, idx_out, dist_out, q, (cudaStream_t)stream,
                 bound);
    FT_API_END
}

// Self-kNN for callers that cannot have device memory allocated for them (see
// fast_self_knn_noalloc in ft_fast.cu): the fast walk's scratch is a fixed static array.
ft_status ft_self_knn_noalloc(ft_context *ctx, const ft_tree *tree, const int32_t *leaf_ids, size_t num, int k,
                              int exclude_self, uint64_t *idx_out, void *dist_out, ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx && tree, "null argument");
    if (!leaf_ids) num = tree->num_leaves;
    if (num > ft::noalloc_max_queries())
        fail(FT_ERR_INVALID_ARGUMENT, "ft_self_knn_noalloc: more than 1048576 queries in one call (the fixed "
                                      "scratch holds 2^20); split the call");
    if (tree->num_leaves == 0 || num == 0 || k <= 0) return FT_OK;
    need(idx_out && dist_out, "null output array");
    if (k > 512) fail(FT_ERR_RUNTIME, "self_knn_query: k too large for shared memory.");
    DeviceGuard g(ctx->device);
    // the kernels write straight into these arrays: pageable host memory would fault there
    need_device(leaf_ids, "leaf_ids");
    need_device(idx_out, "idx_out");
    need_device(dist_out, "dist_out");
    cudaStream_t st = (cudaStream_t)stream;
    if (!ft::fast_self_knn_noalloc(*ctx, *tree, leaf_ids, num, k, exclude_self != 0, idx_out, dist_out, st)) {
        ft_query_options q{}; // reference traversal: it uses no scratch
        q.max_k  = k < 32 ? 32 : k;
        q.method = FT_METHOD_PLAIN;
        ft::self_knn(*ctx, *tree, leaf_ids, num, k, exclude_self != 0, idx_out, dist_out, q, st);
    }
    FT_API_END
}

ft_status ft_knn(ft_context *ctx, const ft_tree *tree, const void *qx, const void *qy, const void *qz,
                 size_t num_queries, int k, uint64_t *idx_out, void *dist_out, const ft_query_options *qopts,
                 ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx && tree, "null argument");
    ft_query_options q{};
    if (qopts) q = *qopts;
    if (tree->num_leaves == 0 || num_queries == 0 || k <= 0) return FT_OK; // src/hlbvh.hpp:1418
    need(qx && qy && qz && idx_out && dist_out, "null argument");
    DeviceGuard  g(ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    size_t       cb = coord_bytes(ctx->opts.coord_type);
    size_t       nk = num_queries * (size_t)k;
    Staged       sx, sy, sz, si, sd;
    sx.init(qx, num_queries * cb, true, false, st);
    sy.init(qy, num_queries * cb, true, false, st);
    sz.init(qz, num_queries * cb, true, false, st);
    si.init(idx_out, nk * 8, false, true, st);
    sd.init(dist_out, nk * 8, false, true, st);
    ft::knn(*ctx, *tree, sx.dev, sy.dev, sz.dev, num_queries, k, q.max_k, (uint64_t *)si.dev, sd.dev, q, st);
    si.copy_back();
    sd.copy_back();
    check_device_status(ctx->status, st);
    FT_API_END
}

ft_status ft_range(ft_context *ctx, const ft_tree *tree, const void *qx, const void *qy, const void *qz,
                   const void *r_min, const void *r_max, size_t num_queries, int32_t *results, int32_t *counts,
                   int max_results_per_query, ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx && tree, "null argument");
    if (tree->num_leaves == 0 || num_queries == 0) return FT_OK; // src/hlbvh.hpp:2020
    need(qx && qy && qz && r_min && r_max && counts, "null argument");
    need(max_results_per_query >= 0, "negative max_results_per_query");
    need(results || max_results_per_query == 0, "null results");
    DeviceGuard  g(ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    size_t       cb = coord_bytes(ctx->opts.coord_type);
    Staged       sx, sy, sz, s0, s1, sr, sc;
    sx.init(qx, num_queries * cb, true, false, st);
    sy.init(qy, num_queries * cb, true, false, st);
    sz.init(qz, num_queries * cb, true, false, st);
    s0.init(r_min, num_queries * cb, true, false, st);
    s1.init(r_max, num_queries * cb, true, false, st);
    // the reference leaves unused result slots untouched: stage with a copy-in
    sr.init(results, num_queries * (size_t)max_results_per_query * 4, true, true, st);
    sc.init(counts, num_queries * 4, false, true, st);
    ft::range(*ctx, *tree, sx.dev, sy.dev, sz.dev, s0.dev, s1.dev, num_queries, (int32_t *)sr.dev, (int32_t *)sc.dev,
              max_results_per_query, st);
    sr.copy_back();
    sc.copy_back();
    check_device_status(ctx->status, st);
    FT_API_END
}

// ---------------------------------------------------------------------------------------
// Learned radius bound (ft_learned.cu)
// ---------------------------------------------------------------------------------------
ft_status ft_bound_model_create(ft_context *ctx, uint64_t seed, ft_bound_model **out) {
    FT_API_BEGIN
    need(ctx && out, "null argument");
    DeviceGuard     g(ctx->device);
    ft::BoundModel *b = ft::bound_model_create(*ctx, seed);
    ft_bound_model *h = new (std::nothrow) ft_bound_model{b};
    if (!h) {
        ft::bound_model_free(b);
        throw std::bad_alloc();
    }
    *out = h;
    FT_API_END
}

ft_status ft_bound_model_destroy(ft_context *ctx, ft_bound_model *model) {
    FT_API_BEGIN
    if (!model) return FT_OK;
    need(ctx != nullptr, "null context");
    DeviceGuard g(ctx->device);
    ft::bound_model_free(model->impl);
    delete model;
    FT_API_END
}

ft_status ft_bound_model_get_params(ft_context *ctx, ft_bound_model *model, float *params_out) {
    FT_API_BEGIN
    need(ctx && model && params_out, "null argument");
    DeviceGuard g(ctx->device);
    ft::bound_model_get_params(*model->impl, params_out);
    FT_API_END
}

ft_status ft_bound_model_set_params(ft_context *ctx, ft_bound_model *model, const float *params) {
    FT_API_BEGIN
    need(ctx && model && params, "null argument");
    DeviceGuard g(ctx->device);
    ft::bound_model_set_params(*model->impl, params, nullptr);
    FT_API_END
}

ft_status ft_bound_model_set_norm(ft_context *ctx, ft_bound_model *model, const float *feature_mean,
                                  const float *feature_std, float target_mean, float target_std) {
    FT_API_BEGIN
    need(ctx && model && feature_mean && feature_std, "null argument");
    DeviceGuard g(ctx->device);
    ft::bound_model_set_norm(*model->impl, feature_mean, feature_std, target_mean, target_std);
    FT_API_END
}

ft_status ft_bound_features(ft_context *ctx, const ft_tree *tree, const int32_t *leaf_ids, size_t num, int k,
                            float *features_out, ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx && tree, "null argument");
    if (!leaf_ids) num = tree->num_leaves;
    need(num <= (size_t)INT32_MAX, "too many queries");
    if (num > 0) need(features_out != nullptr, "null output array");
    need_device(features_out, "features_out");
    DeviceGuard g(ctx->device);
    ft::bound_features(*ctx, *tree, leaf_ids, num, k, features_out, (cudaStream_t)stream);
    FT_API_END
}

ft_status ft_bound_targets(ft_context *ctx, const uint64_t *idx, const void *dist, size_t num, int k,
                           float *targets_out, ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx != nullptr, "null context");
    need(k > 0, "k must be positive");
    need(num <= (size_t)INT32_MAX, "too many rows");
    if (num > 0) need(idx && dist && targets_out, "null array argument");
    DeviceGuard g(ctx->device);
    ft::bound_targets(*ctx, idx, dist, num, k, targets_out, (cudaStream_t)stream);
    FT_API_END
}

ft_status ft_bound_model_gradient(ft_context *ctx, ft_bound_model *model, const float *features,
                                  const float *targets, size_t n, float *grad_out, float *loss_out,
                                  ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx && model && features && targets, "null argument");
    need(n >= 1 && n <= (size_t)(1 << 24), "n must be in [1, 2^24]");
    DeviceGuard g(ctx->device);
    ft::bound_model_gradient(*model->impl, features, targets, (int)n, grad_out, loss_out, (cudaStream_t)stream);
    FT_API_END
}

ft_status ft_bound_model_fit(ft_context *ctx, ft_bound_model *model, const float *features, const float *targets,
                             size_t n, int steps, int batch, float lr, uint64_t seed, float *loss_out,
                             ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx && model && features && targets, "null argument");
    need(n >= 1 && n <= (size_t)INT32_MAX, "n must be in [1, 2^31)");
    need(batch >= 1 && batch <= (1 << 20), "batch must be in [1, 2^20]");
    need(steps >= 0, "negative step count");
    DeviceGuard g(ctx->device);
    ft::bound_model_fit(*model->impl, features, targets, (int)n, steps, batch, lr, seed, loss_out,
                        (cudaStream_t)stream);
    FT_API_END
}

ft_status ft_bound_model_predict(ft_context *ctx, ft_bound_model *model, const float *features, size_t n,
                                 float inflation, float *pred_out, void *bound_out, ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx && model, "null argument");
    need(n <= (size_t)INT32_MAX, "too many rows");
    if (n > 0) need(features != nullptr, "null features");
    DeviceGuard g(ctx->device);
    ft::bound_model_predict(*ctx, *model->impl, features, n, inflation, pred_out, bound_out, (cudaStream_t)stream);
    FT_API_END
}

ft_status ft_bound_features_points(ft_context *ctx, const ft_tree *tree, const void *qx, const void *qy,
                                   const void *qz, size_t num_queries, int k, float *features_out,
                                   ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx && tree, "null argument");
    need(num_queries <= (size_t)INT32_MAX, "too many queries");
    if (num_queries > 0) need(qx && qy && qz && features_out, "null array argument");
    need_device(qx, "qx");
    need_device(qy, "qy");
    need_device(qz, "qz");
    need_device(features_out, "features_out");
    DeviceGuard g(ctx->device);
    ft::bound_features_points(*ctx, *tree, qx, qy, qz, num_queries, k, features_out, (cudaStream_t)stream);
    FT_API_END
}

ft_status ft_knn_learned(ft_context *ctx, const ft_tree *tree, ft_bound_model *model, const void *qx,
                         const void *qy, const void *qz, size_t num_queries, int k, float inflation,
                         uint64_t *idx_out, void *dist_out, const ft_query_options *qopts, ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx && tree && model, "null argument");
    ft_query_options q{};
    if (qopts) q = *qopts;
    if (tree->num_leaves == 0 || num_queries == 0 || k <= 0) return FT_OK;
    need(qx && qy && qz && idx_out && dist_out, "null argument");
    need(num_queries <= (size_t)INT32_MAX, "too many queries");
    const int max_k = q.max_k > 0 ? q.max_k : 256;
    if ((max_k > 32 && k > 32 && k > max_k) || (max_k <= 32 && k > 32))
        fail(FT_ERR_INVALID_ARGUMENT, "k exceeds _MAX_K_ template parameter. Instantiate knn_query with larger _MAX_K_.");
    DeviceGuard  g(ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    size_t       cb = coord_bytes(ctx->opts.coord_type);
    size_t       nk = num_queries * (size_t)k;
    Staged       sx, sy, sz, si, sd;
    sx.init(qx, num_queries * cb, true, false, st);
    sy.init(qy, num_queries * cb, true, false, st);
    sz.init(qz, num_queries * cb, true, false, st);
    si.init(idx_out, nk * 8, false, true, st);
    sd.init(dist_out, nk * 8, false, true, st);
    ft::knn_learned(*ctx, *tree, *model->impl, sx.dev, sy.dev, sz.dev, num_queries, k, max_k, inflation,
                    (uint64_t *)si.dev, sd.dev, q, st);
    si.copy_back();
    sd.copy_back();
    check_device_status(ctx->status, st);
    FT_API_END
}

ft_status ft_self_knn_learned(ft_context *ctx, const ft_tree *tree, ft_bound_model *model, const int32_t *leaf_ids,
                              size_t num, int k, int exclude_self, float inflation, uint64_t *idx_out,
                              void *dist_out, const ft_query_options *qopts, ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx && tree && model, "null argument");
    ft_query_options q{};
    if (qopts) q = *qopts;
    if (!leaf_ids) num = tree->num_leaves;
    need(num <= (size_t)INT32_MAX, "too many queries");
    const int max_k = q.max_k > 0 ? q.max_k : (leaf_ids ? 256 : 32);
    if (k > max_k)
        fail(FT_ERR_INVALID_ARGUMENT,
             "k exceeds _MAX_K_ template parameter. Instantiate self_knn_query with larger _MAX_K_.");
    if (num > 0 && k > 0 && tree->num_leaves > 0) need(idx_out && dist_out, "null output array");
    DeviceGuard g(ctx->device);
    ft::self_knn_learned(*ctx, *tree, *model->impl, leaf_ids, num, k, exclude_self != 0, inflation, idx_out,
                         dist_out, q, (cudaStream_t)stream);
    FT_API_END
}

// ---------------------------------------------------------------------------------------
// Batched sets (ft_batch.cu)
// ---------------------------------------------------------------------------------------
ft_status ft_batch_create(ft_context *ctx, size_t max_points, size_t max_sets, ft_batch **out) {
    FT_API_BEGIN
    need(ctx && out, "null argument");
    DeviceGuard g(ctx->device);
    ft::BatchImpl *b = ft::batch_create(*ctx, max_points, max_sets);
    ft_batch      *h = new (std::nothrow) ft_batch{b};
    if (!h) {
        ft::batch_free(b);
        throw std::bad_alloc();
    }
    *out = h;
    FT_API_END
}

ft_status ft_batch_destroy(ft_context *ctx, ft_batch *batch) {
    FT_API_BEGIN
    if (!batch) return FT_OK;
    need(ctx != nullptr, "null context");
    DeviceGuard g(ctx->device);
    ft::batch_free(batch->impl);
    delete batch;
    FT_API_END
}

static void batch_args(const int64_t *off, size_t num_points, const void *x, const void *y, const void *z,
                       const uint32_t *id, const int8_t *is_ghost) {
    need(off != nullptr, "null set_offsets");
    need(num_points == 0 || (x && y && z), "null coordinate array");
    need_device(off, "set_offsets");
    need_device(x, "x");
    need_device(y, "y");
    need_device(z, "z");
    need_device(id, "id");
    need_device(is_ghost, "is_ghost");
}

ft_status ft_batch_build(ft_context *ctx, ft_batch *batch, const int64_t *set_offsets, size_t num_sets,
                         size_t num_points, const void *x, const void *y, const void *z, const uint32_t *id,
                         const int8_t *is_ghost, ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx && batch, "null argument");
    DeviceGuard g(ctx->device);
    batch_args(set_offsets, num_points, x, y, z, id, is_ghost);
    ft::batch_build(*ctx, *batch->impl, (const long long *)set_offsets, num_sets, num_points, x, y, z, id, is_ghost,
                    (cudaStream_t)stream);
    FT_API_END
}

ft_status ft_batch_set_build_method(ft_context *ctx, ft_batch *batch, int method) {
    FT_API_BEGIN
    need(ctx && batch, "null argument");
    need(method >= FT_METHOD_DEFAULT && method <= FT_METHOD_PERSISTENT, "unknown method");
    ft::batch_set_build_method(*batch->impl, method);
    FT_API_END
}

ft_status ft_batch_self_knn(ft_context *ctx, ft_batch *batch, int k, int exclude_self, uint64_t *idx_out,
                            void *dist_out, const ft_query_options *qopts, ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx && batch, "null argument");
    ft_query_options q{};
    if (qopts) q = *qopts;
    DeviceGuard g(ctx->device);
    if (k > 0) {
        need(idx_out && dist_out, "null output array");
        need_device(idx_out, "idx_out");
        need_device(dist_out, "dist_out");
    }
    ft::batch_query(*ctx, *batch->impl, k, exclude_self != 0, idx_out, dist_out, q, (cudaStream_t)stream);
    FT_API_END
}

ft_status ft_batch_build_knn(ft_context *ctx, ft_batch *batch, const int64_t *set_offsets, size_t num_sets,
                             size_t num_points, const void *x, const void *y, const void *z, const uint32_t *id,
                             const int8_t *is_ghost, int k, int exclude_self, uint64_t *idx_out, void *dist_out,
                             const ft_query_options *qopts, ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx && batch, "null argument");
    ft_query_options q{};
    if (qopts) q = *qopts;
    DeviceGuard g(ctx->device);
    batch_args(set_offsets, num_points, x, y, z, id, is_ghost);
    if (k > 0) {
        need(idx_out && dist_out, "null output array");
        need_device(idx_out, "idx_out");
        need_device(dist_out, "dist_out");
    }
    ft::batch_build_query_graph(*ctx, *batch->impl, (const long long *)set_offsets, num_sets, num_points, x, y, z,
                                id, is_ghost, k, exclude_self != 0, idx_out, dist_out, q, (cudaStream_t)stream);
    FT_API_END
}

ft_status ft_batch_bound_features(ft_context *ctx, ft_batch *batch, int k, float *features_out, ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx && batch, "null argument");
    need_device(features_out, "features_out");
    DeviceGuard g(ctx->device);
    ft::batch_features(*ctx, *batch->impl, k, features_out, (cudaStream_t)stream);
    FT_API_END
}

ft_status ft_batch_self_knn_learned(ft_context *ctx, ft_batch *batch, ft_bound_model *model, int k, int exclude_self,
                                    float inflation, uint64_t *idx_out, void *dist_out, const ft_query_options *qopts,
                                    ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx && batch && model, "null argument");
    need(inflation > 0.0f, "inflation must be positive");
    ft_query_options q{};
    if (qopts) q = *qopts;
    DeviceGuard g(ctx->device);
    if (k > 0) {
        need(idx_out && dist_out, "null output array");
        need_device(idx_out, "idx_out");
        need_device(dist_out, "dist_out");
    }
    ft::batch_query_learned(*ctx, *batch->impl, *model->impl, k, exclude_self != 0, inflation, idx_out, dist_out, q,
                            (cudaStream_t)stream);
    FT_API_END
}

ft_status ft_batch_build_knn_learned(ft_context *ctx, ft_batch *batch, ft_bound_model *model, float inflation,
                                     const int64_t *set_offsets, size_t num_sets, size_t num_points, const void *x,
                                     const void *y, const void *z, const uint32_t *id, const int8_t *is_ghost, int k,
                                     int exclude_self, uint64_t *idx_out, void *dist_out,
                                     const ft_query_options *qopts, ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx && batch && model, "null argument");
    need(inflation > 0.0f, "inflation must be positive");
    need(k <= 64, "learned bound: k must be in [1, 64]");
    ft_query_options q{};
    if (qopts) q = *qopts;
    DeviceGuard g(ctx->device);
    batch_args(set_offsets, num_points, x, y, z, id, is_ghost);
    if (k > 0) {
        need(idx_out && dist_out, "null output array");
        need_device(idx_out, "idx_out");
        need_device(dist_out, "dist_out");
    }
    ft::batch_build_query_graph(*ctx, *batch->impl, (const long long *)set_offsets, num_sets, num_points, x, y, z,
                                id, is_ghost, k, exclude_self != 0, idx_out, dist_out, q, (cudaStream_t)stream,
                                model->impl, inflation);
    FT_API_END
}

// ---------------------------------------------------------------------------------------
// Autotuner (ft_tune.cu)
// ---------------------------------------------------------------------------------------
ft_status ft_tune_self_knn(ft_context *ctx, const ft_tree *tree, int k, int exclude_self, ft_tune_result *out,
                           ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx && tree, "null argument");
    DeviceGuard g(ctx->device);
    ft::tune_self_knn(*ctx, *tree, k, exclude_self != 0, out, (cudaStream_t)stream);
    check_device_status(ctx->status, (cudaStream_t)stream);
    FT_API_END
}

ft_status ft_tune_batch_self_knn(ft_context *ctx, ft_batch *batch, int k, int exclude_self, ft_tune_result *out,
                                 ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx && batch, "null argument");
    DeviceGuard g(ctx->device);
    ft::batch_tune(*ctx, *batch->impl, k, exclude_self != 0, out, (cudaStream_t)stream);
    check_device_status(ctx->status, (cudaStream_t)stream);
    FT_API_END
}

ft_status ft_tune_build(ft_context *ctx, const void *x, const void *y, const void *z, size_t n, ft_tree *tree,
                        ft_tune_result *out, ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx && tree, "null argument");
    need_owned(tree);
    need(x && y && z, "null coordinate array");
    need(n >= 2, "the build autotuner needs 2+ points");
    need(n <= (size_t)(INT_MAX / 2), "Particle count n exceeds maximum supported tree size (INT_MAX / 2).");
    need(tree->capacity >= n, "tree capacity is smaller than the particle count");
    DeviceGuard  g(ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    {
        const size_t cb = coord_bytes(ctx->opts.coord_type);
        Staged       sx, sy, sz;
        sx.init(x, n * cb, true, false, st);
        sy.init(y, n * cb, true, false, st);
        sz.init(z, n * cb, true, false, st);
        tree->num_leaves   = n;
        tree->num_internal = n - 1;
        ft::tune_build(*ctx, *tree, sx.dev, sy.dev, sz.dev, n, out, st);
        check_status_word(*(TreeImpl *)tree->impl, st);
    }
    // leave the tree built the ordinary way (with the chosen tile)
    const ft_status s2 = ft_build_bvh(ctx, x, y, z, n, nullptr, nullptr, nullptr, nullptr, tree, stream);
    if (s2 != FT_OK) return s2;
    FT_API_END
}

ft_status ft_set_range_walk(ft_context *ctx, int walk) {
    FT_API_BEGIN
    need(ctx != nullptr, "null context");
    need(walk >= 0 && walk <= 4, "range walk must be 0 (default), 1 (binary walk per query), 2 (warp-shared), "
                                 "3 (4-wide walk per query) or 4 (the default with every count taken by groups)");
    ctx->range_walk = walk;
    FT_API_END
}

ft_status ft_set_build_profiling(ft_context *ctx, int enable) {
    FT_API_BEGIN
    need(ctx != nullptr, "null context");
    DeviceGuard g(ctx->device);
    if (enable && !ctx->bprof.ev[0])
        for (int i = 0; i < BS_COUNT; ++i) FT_CUDA(cudaEventCreate(&ctx->bprof.ev[i]));
    ctx->bprof.on       = enable != 0;
    ctx->bprof.recorded = false;
    FT_API_END
}

ft_status ft_get_build_profile(ft_context *ctx, ft_build_profile *out) {
    FT_API_BEGIN
    need(ctx && out, "null argument");
    need(ctx->bprof.recorded, "no profiled build on this context (ft_set_build_profiling, then ft_build_bvh)");
    DeviceGuard g(ctx->device);
    FT_CUDA(cudaEventSynchronize(ctx->bprof.ev[BS_RECORDS]));
    float ms[BS_COUNT] = {0};
    for (int i = 1; i < BS_COUNT; ++i)
        FT_CUDA(cudaEventElapsedTime(&ms[i], ctx->bprof.ev[i - 1], ctx->bprof.ev[i]));
    *out             = ft_build_profile{};
    out->bbox_ms     = ms[BS_BBOX];
    out->encode_ms   = ms[BS_ENCODE];
    out->sort_ms     = ms[BS_SORT];
    out->gather_ms   = ms[BS_GATHER];
    out->topology_ms = ms[BS_TOPOLOGY];
    out->refit_ms    = ms[BS_REFIT];
    out->records_ms  = ms[BS_RECORDS];
    float total      = 0.0f;
    FT_CUDA(cudaEventElapsedTime(&total, ctx->bprof.ev[BS_START], ctx->bprof.ev[BS_RECORDS]));
    out->total_ms = total;
    FT_API_END
}

ft_status ft_tune_reset(ft_context *ctx) {
    FT_API_BEGIN
    need(ctx != nullptr, "null context");
    ctx->tuned.clear();
    FT_API_END
}

ft_status ft_batch_tree(ft_context *ctx, ft_batch *batch, size_t set, ft_tree *out, ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx && batch && out, "null argument");
    DeviceGuard g(ctx->device);
    ft::batch_tree_view(*ctx, *batch->impl, set, *out, (cudaStream_t)stream);
    FT_API_END
}

ft_status ft_batch_set_info(ft_context *ctx, ft_batch *batch, void *bbox_out, uint8_t *height_out,
                            ft_stream_t stream) {
    FT_API_BEGIN
    need(ctx && batch, "null argument");
    DeviceGuard g(ctx->device);
    ft::batch_set_info(*ctx, *batch->impl, bbox_out, height_out, (cudaStream_t)stream);
    FT_API_END
}

ft_status ft_batch_query_stats(ft_context *ctx, ft_batch *batch, ft_query_stats *out) {
    FT_API_BEGIN
    need(ctx && batch && out, "null argument");
    DeviceGuard g(ctx->device);
    *out = ft_query_stats{};
    ft::batch_stats(*batch->impl, *out);
    FT_API_END
}

} // extern "C"
