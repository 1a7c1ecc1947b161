// Taylor winding-number batch that allocates no device memory.
//
// Some callers cannot let a library call cudaMalloc / cudaMallocAsync: applications that give a
// fixed device-memory budget to a host engine or plugin framework and account for every byte
// themselves, real-time loops in which an allocation (and the implicit synchronization or pool
// growth it can cause) would stall a frame, and code that replays work while forbidding new
// allocations. gwnb_winding_taylor_batch_f32 allocates its query-ordering scratch per call; this
// variant keeps that scratch in one file-scope device array instead, so the only memory it touches
// is the caller's inputs and outputs, the BVH and moments, and this array.
//
// The array is GWNB_NOALLOC_MAX_QUERIES queries large (about 5.5 MB) and is held by every GPU that
// loads the library until the process exits. All calls share it: two calls whose work overlaps on
// the GPU (different streams without ordering between them) race on it. Each call clears the part
// that must start at zero. The first call on a device looks up the array's device address with
// cudaGetSymbolAddress (once per device, with that device current); make that first call before
// any stream capture.
#include "gwnb_internal.cuh"

#include <cmath>
#include <mutex>

namespace gwnb {

int taylor_batch_in_scratch(taylor_request const &r, std::uint32_t *scratch, std::uint64_t capacity,
                            cudaStream_t s);
std::size_t radix_sort_u32_scratch_words(std::uint64_t n, int key_bits);

namespace {

constexpr std::uint64_t k_capacity = GWNB_NOALLOC_MAX_QUERIES;
// five regions of k_capacity words (codes, sorted codes, order, two sort buffers) plus the sort's
// histograms, tile counters and tile status: 4 passes x (256 + 1 + 256 per sort tile)
constexpr std::uint64_t k_sort_words = 4 * 256 + 4 + 4 * ((k_capacity + k_sort_tile_u32 - 1) / k_sort_tile_u32) * 256;
constexpr std::uint64_t k_scratch_words = 5 * k_capacity + k_sort_words;

static __device__ __align__(256) std::uint32_t g_noalloc_scratch[k_scratch_words];

constexpr int k_max_devices = 64;
std::mutex g_lookup_mutex;
void *g_scratch_address[k_max_devices] = {};

// Device address of g_noalloc_scratch for the current device (host code must not pass the
// symbol itself to a kernel: on the host it only names a stand-in, not device memory).
int scratch_address(std::uint32_t **out) {
    int dev = 0;
    GWNB_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= k_max_devices)
        return set_error(GWNB_INVALID_ARGUMENT, "no-allocation Taylor batch: device ordinal out of range.");
    std::lock_guard<std::mutex> lock(g_lookup_mutex);
    if (g_scratch_address[dev] == nullptr) {
        void *p = nullptr;
        cudaError_t const e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            return set_cuda_error(e, "cudaGetSymbolAddress(no-allocation scratch)");
        g_scratch_address[dev] = p;
    }
    *out = static_cast<std::uint32_t *>(g_scratch_address[dev]);
    return GWNB_OK;
}

bool has(void const *p, std::uint64_t n) { return n == 0 || p != nullptr; }

} // namespace
} // namespace gwnb

using namespace gwnb;

extern "C" int gwnb_winding_taylor_batch_noalloc_f32(const gwnb_bvh4_f32 *b, const gwnb_moment4_f32 *m,
                                                     const float *qx, const float *qy, const float *qz,
                                                     float *out, uint64_t n, float beta,
                                                     const gwnb_taylor_options *opt, gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::query_taylor_noalloc");
    if (radix_sort_u32_scratch_words(k_capacity, 30) > k_sort_words)
        return set_error(GWNB_INTERNAL_ERROR, "no-allocation Taylor batch: scratch layout mismatch.");
    if (n > k_capacity)
        return set_error(GWNB_INVALID_ARGUMENT,
                         "no-allocation Taylor batch: " + std::to_string(n) + " queries exceed its maximum of " +
                             std::to_string(k_capacity) + " per call (GWNB_NOALLOC_MAX_QUERIES).");
    if (b == nullptr || b->revision == 0 || !ref_valid(b->root.reference) || b->primitive_count == 0 ||
        b->primitive_indices == nullptr || b->triangles == nullptr || !has(b->nodes, b->node_count))
        return set_error(GWNB_INVALID_ARGUMENT, "BVH object contains no queryable data.");
    if (ref_internal(b->root.reference) && ref_offset(b->root.reference) >= b->node_count)
        return set_error(GWNB_INVALID_ARGUMENT, "BVH object contains no queryable data.");
    gwnb_taylor_options o{256, 64, 1, GWNB_NEAR_PLAIN, 1e-3f, 0};
    if (opt != nullptr) {
        o = *opt;
        if (o.block_size == 0)
            o.block_size = 256;
        if (o.stack_capacity == 0)
            o.stack_capacity = 64;
    }
    if (o.block_size < 32 || o.block_size > 1024 || (o.block_size % 32) != 0)
        return set_error(GWNB_INVALID_ARGUMENT, "Query batch block size must be a multiple of 32 in [32, 1024].");
    if (o.stack_capacity <= 0)
        return set_error(GWNB_INVALID_ARGUMENT, "Traversal stack capacity must be positive.");
    bool const internal_root = ref_internal(b->root.reference);
    if (internal_root && b->internal_stack_bound > static_cast<std::uint32_t>(o.stack_capacity))
        return set_error(GWNB_INVALID_ARGUMENT, "Traversal stack capacity is below the BVH internal stack bound.");
    if (internal_root && b->internal_stack_bound > 128)
        return set_error(GWNB_INVALID_ARGUMENT, "Traversal stack bounds above 128 are not supported.");
    if (m == nullptr || m->bvh_revision != b->revision ||
        (internal_root ? (m->nodes == nullptr || m->node_count != b->node_count || m->aux == nullptr)
                       : m->node_count != 0))
        return set_error(GWNB_INVALID_ARGUMENT, "Moment object is not aligned with the BVH.");
    if (!(beta >= 0.0f))
        return set_error(GWNB_INVALID_ARGUMENT, "Taylor accuracy scale must be nonnegative.");
    if (o.near_precision != GWNB_NEAR_PLAIN && o.near_precision != GWNB_NEAR_COMPENSATED)
        return set_error(GWNB_INVALID_ARGUMENT, "Unknown near-field precision mode.");
    if (o.per_thread != 0 && o.per_thread != 1)
        return set_error(GWNB_INVALID_ARGUMENT, "Unknown traversal (per_thread must be 0 or 1).");
    if (!has(qx, n) || !has(qy, n) || !has(qz, n) || !has(out, n))
        return set_error(GWNB_INVALID_ARGUMENT, "Query/output spans must use non-null storage when non-empty.");
    // The BVH's derived state must already exist: creating it would allocate.
    auto const *a = reinterpret_cast<bvh_aux_impl const *>(b->aux);
    if (a == nullptr || !a->derived || a->nodes_ptr != b->nodes || a->triangles_ptr != b->triangles ||
        a->node_count != b->node_count || a->primitive_count != b->primitive_count || a->revision != b->revision)
        return set_error(GWNB_INVALID_ARGUMENT,
                         "no-allocation Taylor batch: the BVH lacks current derived state; build or refit it "
                         "with this library (or run one allocating batch) first.");
    if (n == 0)
        return GWNB_OK;
    cudaStream_t const s = reinterpret_cast<cudaStream_t>(stream);
    std::uint32_t *scratch = nullptr;
    GWNB_TRY(scratch_address(&scratch));
    auto const *ma = reinterpret_cast<moment_aux_impl const *>(m->aux);
    taylor_request r{};
    r.order = m->order;
    r.qnodes = ma != nullptr ? ma->qnodes : nullptr;
    r.qcounts = ma != nullptr ? ma->qcounts : nullptr;
    r.tri48 = a->tri48;
    r.primitive_count = b->primitive_count;
    r.node_count = b->node_count;
    r.root_ref = b->root.reference;
    r.root_bounds = a->root_bounds;
    r.qx = qx;
    r.qy = qy;
    r.qz = qz;
    r.out = out;
    r.n = n;
    r.accuracy_scale = beta;
    r.block = o.block_size;
    r.stack_capacity = b->internal_stack_bound > 0 ? static_cast<int>(b->internal_stack_bound) : 1;
    r.sort_queries = o.sort_queries;
    r.near_mode = o.near_precision;
    r.per_thread = o.per_thread;
    r.fp64_threshold = o.fp64_threshold;
    r.fp64_count = a->fp64_count;
    r.status = a->status;
    if (o.near_precision == GWNB_NEAR_COMPENSATED)
        GWNB_CUDA_TRY(cudaMemsetAsync(a->fp64_count, 0, sizeof(unsigned long long), s));
    return taylor_batch_in_scratch(r, scratch, k_capacity, s);
} catch (...) {
    return host_exception();
}
