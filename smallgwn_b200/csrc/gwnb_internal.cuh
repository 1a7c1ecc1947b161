// Internal declarations shared by the libgwnb CUDA translation units.
//
// Layout contract with smallgwn (include/gwn/gwn_bvh.cuh of that project):
//   child = 24 B bounds + 8 B packed reference (bits 0-46 offset, bit 47 valid, 48-63 count),
//   node  = 4 children (128 B), triangle record = {v0, v1 - v0, v2 - v0} (36 B),
//   moment node = field-SoA, one float[4] per field.
// Library-private layouts (query sidecar, padded triangles) are defined here too.
#pragma once

#define GWNB_NVTX_CAT2(a, b) a##b
#define GWNB_NVTX_CAT(a, b) GWNB_NVTX_CAT2(a, b)
#define GWNB_NVTX(name) ::gwnb::nvtx_scope const GWNB_NVTX_CAT(gwnb_nvtx_, __LINE__)(name)

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <tuple>
#include <string>

#include "../../include/gwnb.h"

namespace gwnb {

constexpr std::uint64_t k_offset_mask = (std::uint64_t(1) << 47) - 1;
constexpr std::uint64_t k_valid_bit = std::uint64_t(1) << 47;
constexpr int k_count_shift = 48;
constexpr std::uint32_t k_invalid_u32 = 0xffffffffu;

// Error bits of the device status word that every BVH carries.
enum : unsigned int {
    k_err_index = 1u << 0,        // triangle index out of range
    k_err_topology = 1u << 1,     // inconsistent child references / arrival counts
    k_err_wait_timeout = 1u << 2, // a bounded spin gave up
    k_err_stack_overflow = 1u << 3,
    k_err_collapse = 1u << 4,
    k_err_hploc = 1u << 5,
};

struct aabb {
    float min_x, min_y, min_z, max_x, max_y, max_z;
};
static_assert(sizeof(aabb) == 24);

struct child {
    aabb bounds;
    std::uint64_t reference;
};
static_assert(sizeof(child) == 32);

struct node4 {
    child c[4];
};
static_assert(sizeof(node4) == 128);

struct triangle {
    float v0_x, v0_y, v0_z, e1_x, e1_y, e1_z, e2_x, e2_y, e2_z;
};
static_assert(sizeof(triangle) == 36);

// Padded triangle record for 128-bit loads in traversal: (v0.xyz, e1.x) (e1.yz, e2.xy)
// (e2.z, n.xyz) with n = e1 x e2.
struct alignas(16) triangle48 {
    float4 a, b, c;
};

// The padded record of one triangle: {v0, e1.x | e1.yz, e2.xy | e2.z, n} with n = e1 x e2 in one
// fixed rounding pattern (each component: one product rounded, then one fused multiply-add), so
// every kernel that writes padded records (build, refit, derivation from plain records) stores the
// same bits for the same triangle.
__device__ __forceinline__ triangle48 make_triangle48(float ax, float ay, float az, float e1x, float e1y, float e1z,
                                                      float e2x, float e2y, float e2z) {
    float const nx = __fmaf_rn(e1y, e2z, -__fmul_rn(e1z, e2y));
    float const ny = __fmaf_rn(e1z, e2x, -__fmul_rn(e1x, e2z));
    float const nz = __fmaf_rn(e1x, e2y, -__fmul_rn(e1y, e2x));
    return triangle48{make_float4(ax, ay, az, e1x), make_float4(e1y, e1z, e2x, e2y), make_float4(e2z, nx, ny, nz)};
}

// Sizes of a collapsed BVH4, written by the device for the single read-back that ends a build.
struct collapse_summary {
    unsigned long long node_count;
    std::uint32_t internal_bound;
    std::uint32_t packed_bound;
    std::uint32_t pending; // the levels enqueued did not reach the bottom of the tree
    std::uint32_t pad;
};

struct binary_node {
    std::uint32_t left_index, left_kind, right_index, right_kind;
};
constexpr std::uint32_t k_kind_internal = 1u;
constexpr std::uint32_t k_kind_leaf = 2u;

__host__ __device__ inline bool ref_valid(std::uint64_t r) { return (r & k_valid_bit) != 0; }
__host__ __device__ inline std::uint32_t ref_count(std::uint64_t r) {
    return static_cast<std::uint32_t>(r >> k_count_shift);
}
__host__ __device__ inline bool ref_internal(std::uint64_t r) {
    return ref_valid(r) && ref_count(r) == 0u;
}
__host__ __device__ inline bool ref_leaf(std::uint64_t r) {
    return ref_valid(r) && ref_count(r) != 0u;
}
__host__ __device__ inline std::uint64_t ref_offset(std::uint64_t r) { return r & k_offset_mask; }
__host__ __device__ inline std::uint64_t make_ref(std::uint64_t offset, std::uint64_t count) {
    return k_valid_bit | offset | (count << k_count_shift);
}

// Query sidecar (one record per wide node, written by the moment refit). Per child slot the
// record holds float4 blocks: a = (P.xyz, r2) with r2 < 0 marking an invalid slot,
// b = (N.xyz, ref bits), then the folded far-field coefficients (order 1: the 6 entries of
// M' = trace(M) I - 3M; order 2: those 6 and the 10 of the cubic form K). ref bits: internal child -> node index;
// leaf -> 0x80000000 | first sorted triangle; bit 30 set when the leaf holds more than one
// triangle (its count is then read from the per-node count table).
constexpr std::uint32_t k_qref_leaf = 0x80000000u;
constexpr std::uint32_t k_qref_multi = 0x40000000u;
constexpr std::uint32_t k_qref_index_mask = 0x3fffffffu;

template <int Order> struct qnode_traits;
template <> struct qnode_traits<0> { static constexpr int k_f4_per_child = 2; };
template <> struct qnode_traits<1> { static constexpr int k_f4_per_child = 4; };
template <> struct qnode_traits<2> { static constexpr int k_f4_per_child = 6; };
inline int qnode_f4_per_child(int order) { return order == 0 ? 2 : (order == 1 ? 4 : 6); }

// Field counts of smallgwn's moment node (floats per child slot).
inline int moment_field_count(int order) { return order == 0 ? 7 : (order == 1 ? 13 : 23); }

// Host-side state that travels with a BVH view (gwnb_bvh_aux).
struct bvh_aux_impl {
    bool derived = false;            // parent links / padded triangles are valid for the fields below
    std::uint64_t revision = 0;      // BVH revision this state was derived for
    void *triangles_ptr = nullptr;
    std::uint64_t node_count = 0;
    std::uint64_t primitive_count = 0;
    void *nodes_ptr = nullptr;       // nodes pointer this state was derived for
    // device arrays
    std::uint32_t *parent_slot = nullptr; // (parent << 2) | slot, k_invalid_u32 for the root
    std::uint32_t *expected = nullptr;    // arrivals expected per node
    std::uint32_t *arrivals = nullptr;    // arrival counters (left at zero between calls)
    std::uint32_t *leaf_nodes = nullptr;  // nodes with at least one leaf child
    std::uint64_t leaf_node_count = 0;
    triangle48 *tri48 = nullptr;          // padded triangle records
    aabb *root_bounds = nullptr;          // device copy of the root bounds
    unsigned int *status = nullptr;       // device error word
    unsigned long long *fp64_count = nullptr; // FP64 fallback counter of the compensated path
    void *scratch = nullptr;              // per-BVH reusable scratch for batched queries
    std::size_t scratch_bytes = 0;
    cudaStream_t stream = nullptr;        // stream the arrays were allocated on
};

struct moment_aux_impl {
    float4 *qnodes = nullptr;   // query sidecar, node_count * 4 * f4_per_child float4
    std::uint32_t *qcounts = nullptr; // per node: 4 leaf counts (only read for multi-triangle leaves)
    void *payload = nullptr;    // per-node additive raw-moment payload used by the climb
    std::size_t payload_stride = 0;
};

// ---- host-side validation of C ABI views ----------------------------------------------------------

inline cudaStream_t as_cuda(gwnb_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

inline bool has_storage(void const *p, std::uint64_t n) { return n == 0 || p != nullptr; }

inline bool geometry_valid(gwnb_geometry_f32 const *g) {
    return g != nullptr && has_storage(g->vertex_x, g->vertex_count) &&
           has_storage(g->vertex_y, g->vertex_count) && has_storage(g->vertex_z, g->vertex_count) &&
           has_storage(g->tri_i0, g->triangle_count) && has_storage(g->tri_i1, g->triangle_count) &&
           has_storage(g->tri_i2, g->triangle_count);
}

// A queryable BVH: a revision, a valid root reference and the arrays it implies.
inline bool bvh_valid(gwnb_bvh4_f32 const *b) {
    if (b == nullptr || b->revision == 0 || !ref_valid(b->root.reference) || b->primitive_count == 0)
        return false;
    if (!has_storage(b->nodes, b->node_count) || b->primitive_indices == nullptr || b->triangles == nullptr)
        return false;
    std::uint64_t const off = ref_offset(b->root.reference);
    if (ref_internal(b->root.reference))
        return off < b->node_count;
    std::uint64_t const cnt = ref_count(b->root.reference);
    return off <= b->primitive_count && cnt <= b->primitive_count - off;
}

// Moments refit for exactly this revision of the BVH (smallgwn gwn_bvh_moment_accessor::is_valid_for).
inline bool moment_valid_for(gwnb_moment4_f32 const *m, gwnb_bvh4_f32 const *b) {
    if (m == nullptr || !bvh_valid(b) || m->bvh_revision != b->revision)
        return false;
    if (ref_leaf(b->root.reference))
        return m->node_count == 0;
    return m->nodes != nullptr && m->node_count == b->node_count && m->aux != nullptr;
}

// ---- status helpers (host) -------------------------------------------------------------------
int set_error(int code, std::string const &message);
int set_cuda_error(cudaError_t err, char const *what);
#define GWNB_CUDA_TRY(expr)                                                                        \
    do {                                                                                           \
        cudaError_t gwnb_err_ = (expr);                                                            \
        if (gwnb_err_ != cudaSuccess)                                                              \
            return ::gwnb::set_cuda_error(gwnb_err_, #expr);                                       \
    } while (0)
#define GWNB_TRY(expr)                                                                             \
    do {                                                                                           \
        int gwnb_rc_ = (expr);                                                                     \
        if (gwnb_rc_ != GWNB_OK)                                                                   \
            return gwnb_rc_;                                                                       \
    } while (0)

// The status of a C entry point whose host code threw (std::bad_alloc and the like): no C++
// exception crosses the C ABI; every `int gwnb_*` entry point is a function-try-block ending in it.
int host_exception() noexcept;

std::uint64_t reserve_revision();
int device_sm_count();

// Keys per tile of the 32-bit radix sort (256 threads x 12 keys): callers that size the sort's
// scratch themselves (the allocation-free Taylor batch) use it.
constexpr std::uint64_t k_sort_tile_u32 = 3072;

// A named range on the host timeline (NVTX, header-only): with a profiler attached every library
// call and build or query stage shows as a range around the work it enqueues; without one a
// push / pop is a call through an empty hook.
struct nvtx_scope {
    explicit nvtx_scope(char const *name) { nvtxRangePushA(name); }
    ~nvtx_scope() { nvtxRangePop(); }
    nvtx_scope(nvtx_scope const &) = delete;
    nvtx_scope &operator=(nvtx_scope const &) = delete;
};

template <class F> int nvtx_call(char const *name, F &&f) {
    nvtx_scope const scope(name);
    return f();
}

// Polls after which a device-side wait (the look-back of the radix sort and of the BVH4 collapse)
// gives up, sets k_err_wait_timeout and lets its launch complete. Read by the host when a kernel is
// launched; 2^22 by default, settable with gwnb_set_wait_limit.
constexpr long long k_default_wait_limit = 1ll << 22;
long long wait_limit();

// Counts the kernel launches the library issues (every launch site is `note_launch(), k<<<...>>>`);
// gwnb_launch_count reports the total. A launch recorded into a CUDA graph counts once, at capture.
extern std::atomic<std::uint64_t> g_launch_count;
inline void note_launch() { g_launch_count.fetch_add(1, std::memory_order_relaxed); }

// Threads per block of a query launch. smallgwn's batch configurations accept block sizes up to 1024
// (include/gwn/gwn_query.cuh:37); the query kernels here are compiled for blocks of at most 256
// threads (__launch_bounds__(256): 64 registers per thread at 4 blocks per SM), so a larger request
// launches 256-thread blocks. Every query's result is independent of the block it runs in.
constexpr int k_query_block_max = 256;
inline int query_launch_block(int requested) {
    return requested <= 0 ? k_query_block_max : (requested < k_query_block_max ? requested : k_query_block_max);
}

// Release / acquire fence at GPU scope (PTX fence.acq_rel.gpu). The bottom-up kernels publish a
// node's data with plain stores, this fence, then a relaxed atomic on the node's counter; the
// thread that reads the counter's final value runs this fence before reading the data -- the
// fence-based release/acquire pattern of the PTX memory model. It is cheaper than the sequentially
// consistent __threadfence (fence.sc.gpu), which these patterns do not need.
__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// ---- allocation (stream ordered) ---------------------------------------------------------------
// Every device allocation of the library comes from one memory pool per device that keeps freed
// memory mapped (release threshold at its maximum). With the default pool's threshold of zero,
// each host synchronization hands freed memory back to the driver and the next allocation maps
// it again, which made a 1M-triangle build ~7x slower than its kernels; gwnb_memory_trim returns
// cached memory on request.
int library_pool(cudaMemPool_t *pool);

// Host-side failure injection (gwnb_fail_allocation_after): true when this allocation is the one
// armed to fail; it then reports cudaErrorMemoryAllocation without touching the device.
bool injected_allocation_failure();

template <class T> int alloc(T **ptr, std::size_t count, cudaStream_t s) {
    *ptr = nullptr;
    if (count == 0)
        return GWNB_OK;
    if (injected_allocation_failure())
        return set_cuda_error(cudaErrorMemoryAllocation, "cudaMallocFromPoolAsync (injected failure)");
    cudaMemPool_t pool = nullptr;
    GWNB_TRY(library_pool(&pool));
    void *p = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&p, count * sizeof(T), pool, s);
    if (e != cudaSuccess)
        return set_cuda_error(e, "cudaMallocFromPoolAsync");
    *ptr = static_cast<T *>(p);
    return GWNB_OK;
}
template <class T> void release(T *&ptr, cudaStream_t s) {
    if (ptr != nullptr)
        (void)cudaFreeAsync(ptr, s);
    ptr = nullptr;
}

// The device temporaries of one call: the pointer variables handed to hold() are released on the
// stream when the guard goes out of scope -- on the success path and on every early error return
// alike. A buffer released earlier (release() nulls its pointer) or handed on to an object (null
// the variable) is skipped. Declare the guard after the variables it holds.
class scratch_guard {
public:
    explicit scratch_guard(cudaStream_t s) : s_(s) {}
    scratch_guard(scratch_guard const &) = delete;
    scratch_guard &operator=(scratch_guard const &) = delete;
    ~scratch_guard() {
        for (int i = n_ - 1; i >= 0; --i)
            slots_[i].free_fn(slots_[i].var, s_);
    }
    template <class T> void hold(T *&ptr) {
        if (n_ < k_slots)
            slots_[n_++] = slot{&ptr, &free_var<T>};
    }
    template <class T, class... R> void hold(T *&ptr, R *&...rest) {
        hold(ptr);
        hold(rest...);
    }

private:
    static constexpr int k_slots = 24;
    struct slot {
        void *var;
        void (*free_fn)(void *, cudaStream_t);
    };
    template <class T> static void free_var(void *var, cudaStream_t s) { release(*static_cast<T **>(var), s); }
    slot slots_[k_slots];
    int n_ = 0;
    cudaStream_t s_;
};

// ---- timed walk choice (GWNB_WALK_TIMED) --------------------------------------------------------
// The kind of a batch whose walks are timed against each other: its tree (the moment sidecar for
// Taylor batches, the node array for distance batches), the batch family (0 Taylor, 1 distance),
// and the parameters that change the walk's cost.
struct walk_kind {
    void const *tree;
    int device, family, order, mode, grad, sorted, size_class;
    std::uint32_t scale_bits; // accuracy scale (Taylor) or culling band (distance), as bits
    bool operator<(walk_kind const &o) const {
        return std::tie(tree, device, family, order, mode, grad, sorted, size_class, scale_bits) <
               std::tie(o.tree, o.device, o.family, o.order, o.mode, o.grad, o.sorted, o.size_class, o.scale_bits);
    }
};
struct walk_plan {
    bool per_thread = false;
    cudaEvent_t start = nullptr, stop = nullptr; // recorded around the traversal (null: untimed)
};
// The walk for the next call of kind k on stream s: the first call of a kind walks
// warp-cooperatively and the second per thread, each between two events; later calls take the
// faster once both timings have completed (polled, never waited for). Thread-safe.
walk_plan plan_walk(walk_kind const &k, cudaStream_t s);

// ---- cross-TU kernels / launchers ---------------------------------------------------------------
int radix_sort_pairs(void const *keys_in, void *keys_out, std::uint32_t const *values_in,
                     std::uint32_t *values_out, std::uint64_t n, int key_bytes, int key_bits,
                     cudaStream_t s, unsigned int *status);

// One Taylor / gradient / statistics batch as the C ABI hands it to the query kernels.
struct taylor_request {
    int order;
    float4 const *qnodes;
    std::uint32_t const *qcounts;
    triangle48 const *tri48;
    std::uint64_t primitive_count;
    std::uint64_t node_count;
    std::uint64_t root_ref;
    aabb const *root_bounds; // device
    float const *qx, *qy, *qz;
    float *out, *gx, *gy, *gz;
    std::uint32_t *stat_nodes, *stat_far, *stat_near;
    std::uint64_t n;
    float accuracy_scale;
    int block;
    int stack_capacity; // already >= the BVH's internal stack bound
    int sort_queries;
    int near_mode;
    int per_thread; // 1: one independent traversal per thread; 0: warp-cooperative
    float fp64_threshold;
    unsigned long long *fp64_count;
    unsigned int *status;
    double *probe; // non-null: order the batch and write the sampled-warp probe (6 doubles) instead
};
int taylor_batch(taylor_request const &r, cudaStream_t s);

// One backward pass of the Taylor batch (orders 0 and 1) as the C ABI hands it to the adjoint.
struct adjoint_request {
    int order;
    float4 const *qnodes;
    std::uint32_t const *qcounts;
    triangle48 const *tri48;
    triangle const *triangles;
    node4 const *nodes;
    std::uint64_t primitive_count;
    std::uint64_t node_count;
    std::uint64_t root_ref;
    aabb const *root_bounds;           // device
    std::uint32_t const *parent_slot;  // per node: (parent << 2) | slot
    std::uint32_t const *primitive_indices;
    float const *payload;              // per-node moment payload (area first)
    std::uint64_t payload_floats;
    gwnb_geometry_f32 g;
    float const *qx, *qy, *qz;
    float const *grad_out;
    float *dvx, *dvy, *dvz; // nullptr: no vertex gradients
    float *dqx, *dqy, *dqz; // nullptr: no query gradients
    std::uint64_t n;
    float accuracy_scale;
    int block;
    int stack_capacity;
    int sort_queries;
    unsigned int *status;
};
int taylor_adjoint(adjoint_request const &r, cudaStream_t s);

// Batched refit of many BVHs (bounds, then moments) in one persistent launch each. The device
// descriptor arrays are of types private to the refit translation unit.
struct batch_refit_state {
    std::uint32_t mesh_count = 0;
    int order = 0;
    std::uint64_t bounds_items = 0;
    std::uint64_t moment_items = 0;
    void *bounds_meshes = nullptr;
    void *moment_meshes = nullptr;
    std::uint64_t *bounds_begin = nullptr; // mesh_count + 1 work offsets
    std::uint64_t *moment_begin = nullptr;
};
int batch_refit_prepare(gwnb_geometry_f32 const *geoms, gwnb_bvh4_f32 *const *bvhs, gwnb_moment4_f32 *const *moms,
                        std::uint32_t n, int order, batch_refit_state *st, cudaStream_t s);
int batch_refit_launch(batch_refit_state const &st, int block, bool bounds, bool moments, cudaStream_t s);
void batch_refit_release(batch_refit_state &st, cudaStream_t s);

// Batched Taylor queries of many BVHs in one persistent launch: each mesh's queries occupy a
// range of warp slots (padded to whole warps) of a global slot space.
struct batch_query_state {
    std::uint32_t mesh_count = 0;
    int order = 0;
    int near_mode = GWNB_NEAR_PLAIN;
    std::uint64_t warps = 0;               // total warps of the slot space
    void *meshes = nullptr;                // device per-mesh traversal descriptors (Hilbert order)
    void *meshes_unsorted = nullptr;       // the same in input order
    std::uint64_t *warp_begin = nullptr;   // mesh_count + 1 warp offsets
    std::uint32_t *orders = nullptr;       // per-mesh Hilbert orders, concatenated
    int max_stack_bound = 0;
};
struct batch_query_config {
    int block;      // threads per block (multiple of 32)
    int per_thread; // 0: warp-cooperative traversal, 1: one traversal per thread
    int sorted;     // 1: traverse in each mesh's Hilbert order
    int grid_scale; // persistent grid = SMs x grid_scale blocks
};
int batch_query_prepare(taylor_request const *meshes, std::uint32_t n, batch_query_state *st, cudaStream_t s);
int batch_query_launch(batch_query_state const &st, batch_query_config const &c, cudaStream_t s);
void batch_query_release(batch_query_state &st, cudaStream_t s);

int create_bvh_aux(gwnb_bvh4_f32 *bvh, cudaStream_t s);
int ensure_bvh_aux(gwnb_bvh4_f32 *bvh, cudaStream_t s);
int write_tri48(gwnb_bvh4_f32 const *bvh, cudaStream_t s);

__device__ inline unsigned int lane_id() { return threadIdx.x & 31u; }

// min/max with the operand order of std::min / std::max (keeps signed-zero choices identical).
__host__ __device__ inline float rmin(float a, float b) { return (b < a) ? b : a; }
__host__ __device__ inline float rmax(float a, float b) { return (a < b) ? b : a; }

__device__ inline aabb aabb_union(aabb const &l, aabb const &r) {
    return aabb{rmin(l.min_x, r.min_x), rmin(l.min_y, r.min_y), rmin(l.min_z, r.min_z),
                rmax(l.max_x, r.max_x), rmax(l.max_y, r.max_y), rmax(l.max_z, r.max_z)};
}

// Half surface area with explicit round-to-nearest operations so that the result does not
// depend on floating-point contraction choices.
__device__ inline float aabb_half_area(aabb const &b) {
    float const dx = rmax(__fsub_rn(b.max_x, b.min_x), 0.0f);
    float const dy = rmax(__fsub_rn(b.max_y, b.min_y), 0.0f);
    float const dz = rmax(__fsub_rn(b.max_z, b.min_z), 0.0f);
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dy), __fmul_rn(dy, dz)), __fmul_rn(dz, dx));
}

// Spreads the low 10 bits of v to every third bit.
__device__ inline std::uint32_t expand10(std::uint32_t v) {
    std::uint32_t x = v & 0x3ffu;
    x = (x | (x << 16)) & 0x030000ffu;
    x = (x | (x << 8)) & 0x0300f00fu;
    x = (x | (x << 4)) & 0x030c30c3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

// 30-bit 3D Hilbert index of a point relative to box b (10 bits per axis; the box maps to
// [0.1, 0.9] so points around it spread as well; NaN coordinates map to cell 0). Skilling,
// "Programming the Hilbert curve" (2004): undo the excess work of the Gray-code rotation,
// Gray-encode, then interleave the transposed axes. Consecutive cells are face neighbours, so
// the 32 queries of a warp in this order are more compact than in Morton order.
__device__ inline std::uint32_t hilbert_code30(aabb const &b, float x, float y, float z) {
    float const ex = fmaxf(b.max_x - b.min_x, 1e-30f);
    float const ey = fmaxf(b.max_y - b.min_y, 1e-30f);
    float const ez = fmaxf(b.max_z - b.min_z, 1e-30f);
    auto q = [](float f) -> std::uint32_t {
        f = fminf(fmaxf(f, 0.0f), 1.0f); // NaN -> 0
        return static_cast<std::uint32_t>(f * 1023.0f);
    };
    std::uint32_t X[3] = {q((x - b.min_x) / ex * 0.8f + 0.1f), q((y - b.min_y) / ey * 0.8f + 0.1f),
                          q((z - b.min_z) / ez * 0.8f + 0.1f)};
#pragma unroll
    for (std::uint32_t Q = 1u << 9; Q > 1u; Q >>= 1) {
        std::uint32_t const P = Q - 1u;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            if (X[k] & Q) {
                X[0] ^= P;
            } else {
                std::uint32_t const t = (X[0] ^ X[k]) & P;
                X[0] ^= t;
                X[k] ^= t;
            }
        }
    }
    X[1] ^= X[0];
    X[2] ^= X[1];
    std::uint32_t t = 0;
#pragma unroll
    for (std::uint32_t Q = 1u << 9; Q > 1u; Q >>= 1)
        if (X[2] & Q)
            t ^= Q - 1u;
    return (expand10(X[0] ^ t) << 2) | (expand10(X[1] ^ t) << 1) | expand10(X[2] ^ t);
}

// Loads that bypass L1: data written by other SMs during the same kernel.
__device__ inline float4 ldcg4(float4 const *p) { return __ldcg(p); }

} // namespace gwnb
