// extern "C" entry points of libgwnb (declared in include/gwnb.h).
//
// Validation order and messages follow smallgwn's public functions so status codes line up:
// geometry upload detail/gwn_geometry_impl.cuh:29-206, build detail/gwn_bvh_build_impl.cuh:44-255,
// refit detail/gwn_bvh_refit_impl.cuh:194-334, moment refit
// detail/gwn_bvh_refit_moment_impl.cuh:137-279, queries gwn_query.cuh:308-445.
#include "gwnb_internal.cuh"

#include <atomic>
#include <cmath>
#include <cstring>
#include <exception>
#include <limits>
#include <mutex>
#include <new>
#include <string>

namespace gwnb {

namespace {
thread_local std::string g_message;
thread_local int g_cuda_error = 0;
} // namespace

int set_error(int code, std::string const &message) {
    g_message = message;
    return code;
}

int set_cuda_error(cudaError_t err, char const *what) {
    g_cuda_error = static_cast<int>(err);
    char const *name = cudaGetErrorName(err);
    char const *text = cudaGetErrorString(err);
    g_message = std::string("CUDA API call failed. [cuda_error=") + std::to_string(static_cast<int>(err)) +
                " (" + (name ? name : "unknown") + "): \"" + (text ? text : "unknown") + "\"] in " + what;
    return GWNB_CUDA_RUNTIME_ERROR;
}

std::atomic<std::uint64_t> g_launch_count{0};

namespace {
std::atomic<long long> g_wait_limit{k_default_wait_limit};
} // namespace

long long wait_limit() { return g_wait_limit.load(std::memory_order_relaxed); }

int host_exception() noexcept {
    char const *what = "Unhandled unknown exception.";
    std::string detail;
    try {
        throw;
    } catch (std::bad_alloc const &) {
        what = "Host memory allocation failed.";
    } catch (std::exception const &e) {
        try {
            detail = std::string("Unhandled std::exception: ") + e.what();
        } catch (...) {
        }
    } catch (...) {
    }
    try {
        return set_error(GWNB_INTERNAL_ERROR, detail.empty() ? std::string(what) : detail);
    } catch (...) {
        return GWNB_INTERNAL_ERROR;
    }
}

std::uint64_t reserve_revision() {
    static std::atomic<std::uint64_t> next{1};
    std::uint64_t r = next.load(std::memory_order_relaxed);
    for (;;) {
        if (r == 0 || r == std::numeric_limits<std::uint64_t>::max())
            return 0;
        if (next.compare_exchange_weak(r, r + 1, std::memory_order_relaxed))
            return r;
    }
}

// Allocations left before the injected failure (-1: none armed).
static std::atomic<long long> g_alloc_failure_countdown{-1};

bool injected_allocation_failure() {
    long long c = g_alloc_failure_countdown.load(std::memory_order_relaxed);
    while (c >= 0) {
        if (g_alloc_failure_countdown.compare_exchange_weak(c, c - 1, std::memory_order_relaxed))
            return c == 0;
    }
    return false;
}

int library_pool(cudaMemPool_t *pool) {
    constexpr int k_max_devices = 64;
    static std::mutex mutex;
    static cudaMemPool_t pools[k_max_devices] = {};
    int dev = 0;
    GWNB_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= k_max_devices)
        return set_error(GWNB_INTERNAL_ERROR, "library memory pool: device ordinal out of range.");
    std::lock_guard<std::mutex> lock(mutex);
    if (pools[dev] == nullptr) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t created = nullptr;
        GWNB_CUDA_TRY(cudaMemPoolCreate(&created, &props));
        std::uint64_t keep = std::numeric_limits<std::uint64_t>::max();
        cudaError_t const e = cudaMemPoolSetAttribute(created, cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) {
            (void)cudaMemPoolDestroy(created);
            return set_cuda_error(e, "cudaMemPoolSetAttribute(release threshold)");
        }
        pools[dev] = created;
    }
    *pool = pools[dev];
    return GWNB_OK;
}

int device_sm_count() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess)
        return 148;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
        return 148;
    return sms;
}

// defined in other translation units
int build_preprocess(gwnb_geometry_f32 const &g, int morton_bits, void *sorted_codes,
                     std::uint32_t *sorted_ids, aabb *sorted_aabbs, cudaStream_t s, unsigned int *status);
int build_binary_lbvh(void const *sorted_codes, int morton_bits, std::uint64_t n, aabb const *sorted_aabbs,
                      binary_node *nodes, std::uint32_t *internal_parent, aabb *internal_bounds,
                      cudaStream_t s, unsigned int *status);
int build_binary_hploc(void const *sorted_codes, int morton_bits, std::uint64_t n, aabb const *sorted_aabbs,
                       std::uint32_t radius, binary_node *nodes, std::uint32_t *internal_parent,
                       aabb *internal_bounds, std::uint32_t *root, cudaStream_t s, unsigned int *status,
                       std::uint32_t *counter);
int collapse_to_bvh4(binary_node const *binary, aabb const *binary_bounds, aabb const *leaf_aabbs,
                     std::uint64_t leaf_count, std::uint32_t root_binary, std::uint32_t const *hploc_count,
                     node4 *nodes, std::uint64_t node_capacity, collapse_summary *summary, bool sync,
                     cudaStream_t s, unsigned int *status);
int prepare_bvh_aux_async(gwnb_bvh4_f32 *bvh, std::uint64_t node_capacity, collapse_summary const *summary,
                          std::uint32_t *leaf_node_count, cudaStream_t s);
int onesweep_wait_probe(unsigned int *status, cudaStream_t s);
int collapse_wait_probe(unsigned int *status, cudaStream_t s);
int build_triangles(gwnb_geometry_f32 const &g, std::uint32_t const *ids, std::uint64_t n, triangle *tris,
                    triangle48 *tri48, cudaStream_t s, unsigned int *status);
int refit_bounds_async(gwnb_geometry_f32 const &g, gwnb_bvh4_f32 *bvh, cudaStream_t s);
int refit_moments_async(gwnb_bvh4_f32 const *bvh, gwnb_moment4_f32 *m, cudaStream_t s);
std::size_t moment_payload_bytes(int order);
int exact_batch(triangle const *tris, std::uint64_t nt, float const *qx, float const *qy, float const *qz,
                float *out, std::uint64_t nq, cudaStream_t s);
int exact_batch_f64(gwnb_geometry_f32 const &g, float const *qx, float const *qy, float const *qz, double *out,
                    std::uint64_t nq, cudaStream_t s);
int query_order(aabb const *root_bounds, float const *qx, float const *qy, float const *qz, std::uint64_t n,
                std::uint32_t *order, cudaStream_t s, unsigned int *status);


namespace {

__global__ void k_validate_indices(std::uint32_t const *i0, std::uint32_t const *i1, std::uint32_t const *i2,
                                   std::uint64_t nt, std::uint64_t nv, unsigned int *flag) {
    std::uint64_t const t = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= nt)
        return;
    if (i0[t] >= nv || i1[t] >= nv || i2[t] >= nv)
        atomicExch(flag, 1u);
}

void free_geometry(gwnb_geometry_f32 &g, cudaStream_t s) {
    release(g.tri_i2, s);
    release(g.tri_i1, s);
    release(g.tri_i0, s);
    release(g.vertex_z, s);
    release(g.vertex_y, s);
    release(g.vertex_x, s);
    g.vertex_count = 0;
    g.triangle_count = 0;
}

void free_bvh_aux(gwnb_bvh_aux *&ptr, cudaStream_t s) {
    if (ptr == nullptr)
        return;
    auto *a = reinterpret_cast<bvh_aux_impl *>(ptr);
    release(a->parent_slot, s);
    release(a->expected, s);
    release(a->arrivals, s);
    release(a->leaf_nodes, s);
    release(a->tri48, s);
    release(a->root_bounds, s);
    release(a->status, s);
    release(a->fp64_count, s);
    release(a->scratch, s);
    delete a;
    ptr = nullptr;
}

void free_bvh(gwnb_bvh4_f32 &b, cudaStream_t s) {
    release(b.triangles, s);
    release(b.primitive_indices, s);
    release(b.nodes, s);
    free_bvh_aux(b.aux, s);
    b = gwnb_bvh4_f32{};
}

void free_moment(gwnb_moment4_f32 &m, cudaStream_t s) {
    release(m.nodes, s);
    if (m.aux != nullptr) {
        auto *a = reinterpret_cast<moment_aux_impl *>(m.aux);
        release(a->qnodes, s);
        release(a->qcounts, s);
        release(a->payload, s);
        delete a;
    }
    int const order = m.order;
    m = gwnb_moment4_f32{};
    m.order = order;
}

int read_status(gwnb_bvh4_f32 const *b, unsigned int *out, cudaStream_t s) {
    auto *a = reinterpret_cast<bvh_aux_impl *>(b->aux);
    GWNB_CUDA_TRY(cudaMemcpyAsync(out, a->status, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
    GWNB_CUDA_TRY(cudaStreamSynchronize(s));
    return GWNB_OK;
}

// Device-side results of a build, read back in one copy at its end.
struct build_readback {
    collapse_summary collapse;
    aabb root_bounds;
    unsigned int status;
    std::uint32_t leaf_node_count;
    std::uint32_t hploc_count;
    std::uint32_t pad;
};

// A failing CUDA call inside build_impl releases the staged tree and the temporaries (fail()).
#define GWNB_BUILD_CUDA_TRY(expr)                                                                  \
    do {                                                                                           \
        cudaError_t const gwnb_e_ = (expr);                                                        \
        if (gwnb_e_ != cudaSuccess)                                                                \
            return fail(set_cuda_error(gwnb_e_, #expr));                                           \
    } while (0)

// The build enqueues every stage on the stream without a host round trip (the H-PLOC convergence
// check, the collapse's depth and node count, the leaf-node list of the refit state all stay on
// the device) and synchronizes once, to read the tree's sizes, bounds and error word.
int build_impl(gwnb_geometry_f32 const *g, int method, std::uint32_t radius, int morton_bits,
               gwnb_bvh4_f32 *out, cudaStream_t s) {
    std::uint64_t const nt = g->triangle_count;
    gwnb_bvh4_f32 b{};
    if (int const arc = create_bvh_aux(&b, s); arc != GWNB_OK) {
        free_bvh(b, s);
        return arc;
    }
    auto *aux = reinterpret_cast<bvh_aux_impl *>(b.aux);
    unsigned int *status = aux->status;
    int rc = GWNB_OK;
    void *codes = nullptr;
    aabb *sorted_aabbs = nullptr;
    binary_node *bin = nullptr;
    std::uint32_t *bin_parent = nullptr;
    aabb *bin_bounds = nullptr;
    build_readback *rb = nullptr;
    auto cleanup = [&]() {
        release(codes, s);
        release(sorted_aabbs, s);
        release(bin, s);
        release(bin_parent, s);
        release(bin_bounds, s);
        release(rb, s);
    };
    auto fail = [&](int code) {
        cleanup();
        free_bvh(b, s);
        return code;
    };
    b.primitive_count = nt;
    if ((rc = alloc(&b.primitive_indices, nt, s)) != GWNB_OK)
        return fail(rc);
    if ((rc = alloc(reinterpret_cast<triangle **>(&b.triangles), nt, s)) != GWNB_OK)
        return fail(rc);
    if ((rc = alloc(reinterpret_cast<unsigned char **>(&codes), nt * (morton_bits / 8), s)) != GWNB_OK)
        return fail(rc);
    if ((rc = alloc(&sorted_aabbs, nt, s)) != GWNB_OK)
        return fail(rc);
    if ((rc = alloc(&rb, 1, s)) != GWNB_OK)
        return fail(rc);
    GWNB_BUILD_CUDA_TRY(cudaMemsetAsync(rb, 0, sizeof(build_readback), s));
    if ((rc = nvtx_call("gwnb::build.morton_sort", [&] {
             return build_preprocess(*g, morton_bits, codes, b.primitive_indices, sorted_aabbs, s, status);
         })) != GWNB_OK)
        return fail(rc);
    std::uint64_t capacity = 0;
    std::uint32_t root_binary = 0;
    if (nt == 1) {
        GWNB_BUILD_CUDA_TRY(cudaMemcpyAsync(&rb->root_bounds, sorted_aabbs, sizeof(aabb), cudaMemcpyDeviceToDevice, s));
        b.root.reference = make_ref(0, 1);
    } else {
        std::uint64_t const ni = nt - 1;
        if ((rc = alloc(&bin, ni, s)) != GWNB_OK || (rc = alloc(&bin_parent, ni, s)) != GWNB_OK ||
            (rc = alloc(&bin_bounds, ni, s)) != GWNB_OK)
            return fail(rc);
        root_binary = 0;
        std::uint32_t *hploc_count = nullptr;
        if (method == GWNB_METHOD_LBVH) {
            rc = nvtx_call("gwnb::build.binary_lbvh", [&] {
                return build_binary_lbvh(codes, morton_bits, nt, sorted_aabbs, bin, bin_parent, bin_bounds, s, status);
            });
        } else {
            hploc_count = &rb->hploc_count;
            rc = nvtx_call("gwnb::build.binary_hploc", [&] {
                return build_binary_hploc(codes, morton_bits, nt, sorted_aabbs, radius, bin, bin_parent, bin_bounds,
                                          &root_binary, s, status, hploc_count);
            });
        }
        if (rc != GWNB_OK)
            return fail(rc);
        GWNB_BUILD_CUDA_TRY(cudaMemcpyAsync(&rb->root_bounds, bin_bounds + root_binary, sizeof(aabb),
                                      cudaMemcpyDeviceToDevice, s));
        if ((rc = alloc(reinterpret_cast<node4 **>(&b.nodes), ni, s)) != GWNB_OK)
            return fail(rc);
        b.node_capacity = ni;
        capacity = ni;
        if ((rc = nvtx_call("gwnb::build.collapse", [&] {
                 return collapse_to_bvh4(bin, bin_bounds, sorted_aabbs, nt, root_binary, hploc_count,
                                         reinterpret_cast<node4 *>(b.nodes), ni, &rb->collapse, false, s, status);
             })) != GWNB_OK)
            return fail(rc);
        b.root.reference = make_ref(0, 0);
    }
    // refit / query state: parent links and leaf-node list over the collapsed nodes (sized by the
    // node capacity; the kernels read the node count from the device), padded triangle records
    // written with the leaf-ordered ones
    if ((rc = nvtx_call("gwnb::build.records", [&] {
             int const prc = prepare_bvh_aux_async(&b, capacity, &rb->collapse, &rb->leaf_node_count, s);
             return prc != GWNB_OK ? prc
                                   : build_triangles(*g, b.primitive_indices, nt,
                                                     reinterpret_cast<triangle *>(b.triangles), aux->tri48, s, status);
         })) != GWNB_OK)
        return fail(rc);
    GWNB_BUILD_CUDA_TRY(cudaMemcpyAsync(aux->root_bounds, &rb->root_bounds, sizeof(aabb), cudaMemcpyDeviceToDevice, s));
    GWNB_BUILD_CUDA_TRY(cudaMemcpyAsync(&rb->status, status, sizeof(unsigned int), cudaMemcpyDeviceToDevice, s));
    build_readback host{};
    GWNB_BUILD_CUDA_TRY(cudaMemcpyAsync(&host, rb, sizeof(host), cudaMemcpyDeviceToHost, s));
    GWNB_BUILD_CUDA_TRY(cudaStreamSynchronize(s));
    if (host.status == 0u && nt > 1 && host.collapse.pending != 0u) {
        // a tree deeper than the levels enqueued up front: collapse again level batch by level batch,
        // then derive the refit state again from the complete nodes
        if ((rc = collapse_to_bvh4(bin, bin_bounds, sorted_aabbs, nt, root_binary, nullptr,
                                   reinterpret_cast<node4 *>(b.nodes), capacity, &rb->collapse, true, s, status)) !=
            GWNB_OK)
            return fail(rc);
        if ((rc = prepare_bvh_aux_async(&b, capacity, &rb->collapse, &rb->leaf_node_count, s)) != GWNB_OK)
            return fail(rc);
        if ((rc = build_triangles(*g, b.primitive_indices, nt, reinterpret_cast<triangle *>(b.triangles), aux->tri48,
                                  s, status)) != GWNB_OK)
            return fail(rc);
        GWNB_BUILD_CUDA_TRY(cudaMemcpyAsync(&rb->status, status, sizeof(unsigned int), cudaMemcpyDeviceToDevice, s));
        GWNB_BUILD_CUDA_TRY(cudaMemcpyAsync(&host, rb, sizeof(host), cudaMemcpyDeviceToHost, s));
        GWNB_BUILD_CUDA_TRY(cudaStreamSynchronize(s));
    }
    if (host.status != 0u) {
        if (host.status & k_err_index)
            return fail(set_error(GWNB_INTERNAL_ERROR,
                                  "bvh.build: Leaf-ordered triangle construction encountered invalid geometry."));
        if (host.status & k_err_hploc)
            return fail(set_error(GWNB_INTERNAL_ERROR,
                                  "bvh.build.binary.hploc: H-PLOC builder did not converge to a complete binary hierarchy."));
        return fail(set_error(GWNB_INTERNAL_ERROR, "bvh.build: device builder reported an inconsistent hierarchy (status " +
                                                       std::to_string(host.status) + ")."));
    }
    if (nt > 1) {
        b.node_count = host.collapse.node_count;
        b.internal_stack_bound = host.collapse.internal_bound;
        b.packed_stack_bound = host.collapse.packed_bound;
        if (b.node_count == 0)
            return fail(set_error(GWNB_INTERNAL_ERROR, "bvh.build.collapse: collapse produced no nodes."));
    }
    aux->leaf_node_count = host.leaf_node_count;
    std::memcpy(&b.root.bounds, &host.root_bounds, sizeof(aabb));
    cleanup();
    b.revision = reserve_revision();
    if (b.revision == 0)
        return fail(set_error(GWNB_INTERNAL_ERROR, "bvh.build: BVH geometry-derived state revision is exhausted."));
    aux->nodes_ptr = b.nodes;
    aux->triangles_ptr = b.triangles;
    aux->node_count = b.node_count;
    aux->primitive_count = b.primitive_count;
    aux->revision = b.revision;
    aux->derived = true;
    *out = b;
    return GWNB_OK;
}
#undef GWNB_BUILD_CUDA_TRY

} // namespace
} // namespace gwnb

using namespace gwnb;

extern "C" {

const char *gwnb_last_error_message(void) { return g_message.c_str(); }

uint64_t gwnb_launch_count(void) { return g_launch_count.load(std::memory_order_relaxed); }

int gwnb_memory_stats(uint64_t *reserved, uint64_t *used) try {
    cudaMemPool_t pool = nullptr;
    GWNB_TRY(library_pool(&pool));
    std::uint64_t r = 0, u = 0;
    GWNB_CUDA_TRY(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &r));
    GWNB_CUDA_TRY(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &u));
    if (reserved != nullptr)
        *reserved = r;
    if (used != nullptr)
        *used = u;
    return GWNB_OK;
} catch (...) {
    return host_exception();
}

int gwnb_set_wait_limit(int64_t polls) try {
    g_wait_limit.store(polls > 0 ? static_cast<long long>(polls) : k_default_wait_limit, std::memory_order_relaxed);
    return GWNB_OK;
} catch (...) {
    return host_exception();
}

int gwnb_wait_timeout_probe(int stage, gwnb_stream_t stream) try {
    if (stage != 0 && stage != 1)
        return set_error(GWNB_INVALID_ARGUMENT, "wait probe: stage must be 0 (radix sort) or 1 (BVH4 collapse).");
    cudaStream_t const s = as_cuda(stream);
    unsigned int *status = nullptr;
    GWNB_TRY(alloc(&status, 1, s));
    int rc = GWNB_OK;
    if (cudaMemsetAsync(status, 0, sizeof(unsigned int), s) != cudaSuccess)
        rc = set_cuda_error(cudaGetLastError(), "wait probe status");
    if (rc == GWNB_OK)
        rc = stage == 0 ? onesweep_wait_probe(status, s) : collapse_wait_probe(status, s);
    unsigned int host = 0;
    if (rc == GWNB_OK) {
        cudaError_t e = cudaMemcpyAsync(&host, status, sizeof(host), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(s);
        if (e != cudaSuccess)
            rc = set_cuda_error(e, "wait probe status read-back");
    }
    release(status, s);
    if (rc != GWNB_OK)
        return rc;
    if (host & k_err_wait_timeout)
        return set_error(GWNB_INTERNAL_ERROR, std::string(stage == 0 ? "radix sort" : "BVH4 collapse") +
                                                  ": device wait timed out (predecessor tile never published).");
    return GWNB_OK;
} catch (...) {
    return host_exception();
}

int64_t gwnb_fail_allocation_after(int64_t count) {
    return g_alloc_failure_countdown.exchange(count >= 0 ? count : -1, std::memory_order_relaxed);
}

int gwnb_memory_trim(uint64_t keep_bytes) try {
    cudaMemPool_t pool = nullptr;
    GWNB_TRY(library_pool(&pool));
    GWNB_CUDA_TRY(cudaMemPoolTrimTo(pool, static_cast<std::size_t>(keep_bytes)));
    return GWNB_OK;
} catch (...) {
    return host_exception();
}
int gwnb_last_cuda_error(void) { return g_cuda_error; }
const char *gwnb_version(void) { return "gwnb 0.1 (sm_100a)"; }

int gwnb_cuda_runtime_version(void) {
    int v = 0;
    return cudaRuntimeGetVersion(&v) == cudaSuccess ? v : 0;
}

int gwnb_geometry_upload_f32(gwnb_geometry_f32 *out, const float *x, const float *y, const float *z,
                             uint64_t nv, const uint32_t *i0, const uint32_t *i1, const uint32_t *i2,
                             uint64_t nt, gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::upload_geometry");
    if (out == nullptr)
        return set_error(GWNB_INVALID_ARGUMENT, "gwnb_geometry_upload_f32 requires an output view.");
    if (nv > std::numeric_limits<std::uint32_t>::max())
        return set_error(GWNB_INVALID_ARGUMENT, "Vertex count exceeds index type capacity.");
    if (nt > std::numeric_limits<std::uint32_t>::max())
        return set_error(GWNB_INVALID_ARGUMENT, "Triangle count exceeds index type capacity.");
    if (!has_storage(x, nv) || !has_storage(y, nv) || !has_storage(z, nv) || !has_storage(i0, nt) ||
        !has_storage(i1, nt) || !has_storage(i2, nt))
        return set_error(GWNB_INVALID_ARGUMENT, "Geometry spans must use non-null storage when non-empty.");
    cudaStream_t const s = as_cuda(stream);
    gwnb_geometry_f32 g{};
    int rc = GWNB_OK;
    auto fail = [&](int code) {
        free_geometry(g, s);
        return code;
    };
    if ((rc = alloc(&g.vertex_x, nv, s)) || (rc = alloc(&g.vertex_y, nv, s)) || (rc = alloc(&g.vertex_z, nv, s)) ||
        (rc = alloc(&g.tri_i0, nt, s)) || (rc = alloc(&g.tri_i1, nt, s)) || (rc = alloc(&g.tri_i2, nt, s)))
        return fail(rc);
    g.vertex_count = nv;
    g.triangle_count = nt;
    cudaError_t e = cudaSuccess;
    if (nv > 0) {
        if ((e = cudaMemcpyAsync(g.vertex_x, x, nv * 4, cudaMemcpyDefault, s)) != cudaSuccess ||
            (e = cudaMemcpyAsync(g.vertex_y, y, nv * 4, cudaMemcpyDefault, s)) != cudaSuccess ||
            (e = cudaMemcpyAsync(g.vertex_z, z, nv * 4, cudaMemcpyDefault, s)) != cudaSuccess)
            return fail(set_cuda_error(e, "cudaMemcpyAsync(vertices)"));
    }
    if (nt > 0) {
        if ((e = cudaMemcpyAsync(g.tri_i0, i0, nt * 4, cudaMemcpyDefault, s)) != cudaSuccess ||
            (e = cudaMemcpyAsync(g.tri_i1, i1, nt * 4, cudaMemcpyDefault, s)) != cudaSuccess ||
            (e = cudaMemcpyAsync(g.tri_i2, i2, nt * 4, cudaMemcpyDefault, s)) != cudaSuccess)
            return fail(set_cuda_error(e, "cudaMemcpyAsync(indices)"));
        if (nv == 0)
            return fail(set_error(GWNB_INVALID_ARGUMENT, "Triangle indices require non-empty vertex arrays."));
        unsigned int *flag = nullptr;
        if ((rc = alloc(&flag, 1, s)) != GWNB_OK)
            return fail(rc);
        unsigned int host_flag = 0;
        if ((e = cudaMemsetAsync(flag, 0, sizeof(unsigned int), s)) != cudaSuccess)
            return fail(set_cuda_error(e, "cudaMemsetAsync"));
        note_launch(), k_validate_indices<<<static_cast<unsigned>((nt + 255) / 256), 256, 0, s>>>(g.tri_i0, g.tri_i1, g.tri_i2, nt,
                                                                                 nv, flag);
        if ((e = cudaGetLastError()) != cudaSuccess ||
            (e = cudaMemcpyAsync(&host_flag, flag, sizeof(host_flag), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (e = cudaStreamSynchronize(s)) != cudaSuccess) {
            release(flag, s);
            return fail(set_cuda_error(e, "index validation"));
        }
        release(flag, s);
        if (host_flag != 0)
            return fail(set_error(GWNB_INVALID_ARGUMENT, "Triangle indices must be in [0, vertex_count)."));
    }
    *out = g;
    return GWNB_OK;
} catch (...) {
    return host_exception();
}

static int update_common(gwnb_geometry_f32 *g, const float *x, const float *y, const float *z, uint64_t nv,
                         gwnb_stream_t stream, cudaMemcpyKind kind) {
    if (!geometry_valid(g))
        return set_error(GWNB_INVALID_ARGUMENT, "Geometry accessor is invalid for update.");
    if (nv != g->vertex_count)
        return set_error(GWNB_INVALID_ARGUMENT, "Updated vertex count must match geometry.");
    if (!has_storage(x, nv) || !has_storage(y, nv) || !has_storage(z, nv))
        return set_error(GWNB_INVALID_ARGUMENT, "Geometry update spans must use non-null storage when non-empty.");
    if (nv == 0)
        return GWNB_OK;
    cudaStream_t const s = as_cuda(stream);
    GWNB_CUDA_TRY(cudaMemcpyAsync(g->vertex_x, x, nv * 4, kind, s));
    GWNB_CUDA_TRY(cudaMemcpyAsync(g->vertex_y, y, nv * 4, kind, s));
    GWNB_CUDA_TRY(cudaMemcpyAsync(g->vertex_z, z, nv * 4, kind, s));
    return GWNB_OK;
}

int gwnb_geometry_update_f32(gwnb_geometry_f32 *g, const float *x, const float *y, const float *z, uint64_t nv,
                             gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::update_geometry");
    return update_common(g, x, y, z, nv, stream, cudaMemcpyDefault);
} catch (...) {
    return host_exception();
}

int gwnb_geometry_update_device_f32(gwnb_geometry_f32 *g, const float *x, const float *y, const float *z,
                                    uint64_t nv, gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::update_geometry");
    return update_common(g, x, y, z, nv, stream, cudaMemcpyDeviceToDevice);
} catch (...) {
    return host_exception();
}

void gwnb_geometry_release_f32(gwnb_geometry_f32 *g, gwnb_stream_t stream) {
    if (g != nullptr)
        free_geometry(*g, as_cuda(stream));
}

int gwnb_bvh4_build_f32(const gwnb_geometry_f32 *g, int method, uint32_t radius, int morton_bits,
                        gwnb_bvh4_f32 *out, gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::bvh_build");
    if (out == nullptr)
        return set_error(GWNB_INVALID_ARGUMENT, "bvh.build: output view is null.");
    if (!geometry_valid(g))
        return set_error(GWNB_INVALID_ARGUMENT, "bvh.build: Geometry accessor is invalid for BVH build.");
    if (method != GWNB_METHOD_HPLOC && method != GWNB_METHOD_LBVH)
        return set_error(GWNB_INVALID_ARGUMENT, "bvh.build: BVH build method is invalid.");
    if (method == GWNB_METHOD_HPLOC && (radius == 0 || radius > 8))
        return set_error(GWNB_INVALID_ARGUMENT, "bvh.build: H-PLOC search radius must be in the range [1, 8].");
    if (morton_bits != 32 && morton_bits != 64)
        return set_error(GWNB_INVALID_ARGUMENT, "bvh.build: unsupported instantiation (MortonCode must be uint32 or uint64).");
    std::uint64_t const nt = g->triangle_count;
    if (nt > std::numeric_limits<std::uint32_t>::max())
        return set_error(GWNB_INVALID_ARGUMENT, "bvh.build: Triangle count exceeds the selected BVH index range.");
    if (nt != 0 && g->vertex_count == 0)
        return set_error(GWNB_INVALID_ARGUMENT, "bvh.build: Cannot build a BVH with triangles but no vertices.");
    if (nt >= (std::uint64_t(1) << 30))
        return set_error(GWNB_INVALID_ARGUMENT, "bvh.build: at most 2^30 - 1 triangles are supported.");
    if (nt == 0) {
        *out = gwnb_bvh4_f32{};
        return GWNB_OK;
    }
    return build_impl(g, method, radius, morton_bits, out, as_cuda(stream));
} catch (...) {
    return host_exception();
}

void gwnb_bvh4_release_f32(gwnb_bvh4_f32 *b, gwnb_stream_t stream) {
    if (b != nullptr)
        free_bvh(*b, as_cuda(stream));
}

int gwnb_build_preprocess_f32(const gwnb_geometry_f32 *g, int morton_bits, void *sorted_codes, uint32_t *sorted_ids,
                              gwnb_aabb_f32 *sorted_aabbs, gwnb_stream_t stream) try {
    if (!geometry_valid(g))
        return set_error(GWNB_INVALID_ARGUMENT, "bvh.build.preprocess: geometry is invalid.");
    if (morton_bits != 32 && morton_bits != 64)
        return set_error(GWNB_INVALID_ARGUMENT, "bvh.build.preprocess: morton_bits must be 32 or 64.");
    cudaStream_t const s = as_cuda(stream);
    unsigned int *status = nullptr;
    GWNB_TRY(alloc(&status, 1, s));
    GWNB_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(unsigned int), s));
    int rc = build_preprocess(*g, morton_bits, sorted_codes, sorted_ids, reinterpret_cast<aabb *>(sorted_aabbs), s,
                              status);
    unsigned int host = 0;
    if (rc == GWNB_OK) {
        GWNB_CUDA_TRY(cudaMemcpyAsync(&host, status, sizeof(host), cudaMemcpyDeviceToHost, s));
        GWNB_CUDA_TRY(cudaStreamSynchronize(s));
    }
    release(status, s);
    if (rc == GWNB_OK && host != 0)
        return set_error(GWNB_INTERNAL_ERROR, "bvh.build.preprocess: device sort reported an error.");
    return rc;
} catch (...) {
    return host_exception();
}

int gwnb_build_binary_lbvh(const void *sorted_codes, int morton_bits, uint64_t n, const gwnb_aabb_f32 *sorted_aabbs,
                           gwnb_binary_node *nodes, uint32_t *internal_parent, gwnb_aabb_f32 *internal_bounds,
                           gwnb_stream_t stream) try {
    if (morton_bits != 32 && morton_bits != 64)
        return set_error(GWNB_INVALID_ARGUMENT, "bvh.build.binary.lbvh: morton_bits must be 32 or 64.");
    cudaStream_t const s = as_cuda(stream);
    unsigned int *status = nullptr;
    GWNB_TRY(alloc(&status, 1, s));
    GWNB_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(unsigned int), s));
    int rc = build_binary_lbvh(sorted_codes, morton_bits, n, reinterpret_cast<aabb const *>(sorted_aabbs),
                               reinterpret_cast<binary_node *>(nodes), internal_parent,
                               reinterpret_cast<aabb *>(internal_bounds), s, status);
    unsigned int host = 0;
    if (rc == GWNB_OK) {
        GWNB_CUDA_TRY(cudaMemcpyAsync(&host, status, sizeof(host), cudaMemcpyDeviceToHost, s));
        GWNB_CUDA_TRY(cudaStreamSynchronize(s));
    }
    release(status, s);
    if (rc == GWNB_OK && host != 0)
        return set_error(GWNB_INTERNAL_ERROR, "bvh.build.binary.lbvh: device builder reported an error.");
    return rc;
} catch (...) {
    return host_exception();
}

int gwnb_build_binary_hploc(const void *sorted_codes, int morton_bits, uint64_t n, const gwnb_aabb_f32 *sorted_aabbs,
                            uint32_t radius, gwnb_binary_node *nodes, uint32_t *internal_parent,
                            gwnb_aabb_f32 *internal_bounds, uint32_t *root, gwnb_stream_t stream) try {
    if (morton_bits != 32 && morton_bits != 64)
        return set_error(GWNB_INVALID_ARGUMENT, "bvh.build.binary.hploc: morton_bits must be 32 or 64.");
    if (radius == 0 || radius > 8)
        return set_error(GWNB_INVALID_ARGUMENT, "bvh.build.binary.hploc: H-PLOC search radius must be in the range [1, 8].");
    if (root == nullptr)
        return set_error(GWNB_INVALID_ARGUMENT, "bvh.build.binary.hploc: root output is null.");
    cudaStream_t const s = as_cuda(stream);
    unsigned int *status = nullptr;
    GWNB_TRY(alloc(&status, 1, s));
    GWNB_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(unsigned int), s));
    int const rc = build_binary_hploc(sorted_codes, morton_bits, n, reinterpret_cast<aabb const *>(sorted_aabbs), radius,
                                      reinterpret_cast<binary_node *>(nodes), internal_parent,
                                      reinterpret_cast<aabb *>(internal_bounds), root, s, status, nullptr);
    release(status, s);
    return rc;
} catch (...) {
    return host_exception();
}

int gwnb_radix_sort_pairs(const void *keys_in, void *keys_out, const uint32_t *values_in, uint32_t *values_out,
                          uint64_t count, int key_bytes, int key_bits, gwnb_stream_t stream) try {
    if (count > 0 && (keys_in == nullptr || keys_out == nullptr || values_out == nullptr))
        return set_error(GWNB_INVALID_ARGUMENT, "radix sort: null buffer.");
    cudaStream_t const s = as_cuda(stream);
    unsigned int *status = nullptr;
    GWNB_TRY(alloc(&status, 1, s));
    GWNB_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(unsigned int), s));
    int rc = radix_sort_pairs(keys_in, keys_out, values_in, values_out, count, key_bytes, key_bits, s, status);
    unsigned int host = 0;
    if (rc == GWNB_OK) {
        GWNB_CUDA_TRY(cudaMemcpyAsync(&host, status, sizeof(host), cudaMemcpyDeviceToHost, s));
        GWNB_CUDA_TRY(cudaStreamSynchronize(s));
    }
    release(status, s);
    if (rc == GWNB_OK && host != 0)
        return set_error(GWNB_INTERNAL_ERROR, "radix sort: device look-back timed out.");
    return rc;
} catch (...) {
    return host_exception();
}

// ---- refit --------------------------------------------------------------------------------------

int gwnb_bvh4_refit_async_f32(const gwnb_geometry_f32 *g, gwnb_bvh4_f32 *b, gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::refit_bvh_async");
    if (!geometry_valid(g))
        return set_error(GWNB_INVALID_ARGUMENT, "bvh.refit: Geometry accessor is invalid.");
    if (!bvh_valid(b))
        return set_error(GWNB_INVALID_ARGUMENT, "bvh.refit: BVH accessor is invalid.");
    if (g->triangle_count != b->primitive_count)
        return set_error(GWNB_INVALID_ARGUMENT, "bvh.refit: Geometry triangle count differs from the BVH primitive order.");
    std::uint64_t const next = reserve_revision();
    if (next == 0)
        return set_error(GWNB_INTERNAL_ERROR, "bvh.refit: BVH geometry-derived state revision is exhausted.");
    cudaStream_t const s = as_cuda(stream);
    GWNB_TRY(ensure_bvh_aux(b, s));
    b->revision = 0; // unqueryable until the writes below complete successfully
    GWNB_TRY(refit_bounds_async(*g, b, s));
    b->revision = next;
    reinterpret_cast<bvh_aux_impl *>(b->aux)->revision = next;
    return GWNB_OK;
} catch (...) {
    return host_exception();
}

int gwnb_bvh4_sync_status_f32(gwnb_bvh4_f32 *b, gwnb_stream_t stream) try {
    if (b == nullptr || b->aux == nullptr)
        return set_error(GWNB_INVALID_ARGUMENT, "bvh.status: BVH has no device state.");
    cudaStream_t const s = as_cuda(stream);
    auto *a = reinterpret_cast<bvh_aux_impl *>(b->aux);
    unsigned int host = 0;
    aabb rb{};
    GWNB_CUDA_TRY(cudaMemcpyAsync(&host, a->status, sizeof(host), cudaMemcpyDeviceToHost, s));
    GWNB_CUDA_TRY(cudaMemcpyAsync(&rb, a->root_bounds, sizeof(rb), cudaMemcpyDeviceToHost, s));
    GWNB_CUDA_TRY(cudaStreamSynchronize(s));
    if (host != 0u) {
        GWNB_CUDA_TRY(cudaMemsetAsync(a->status, 0, sizeof(unsigned int), s));
        if (a->arrivals != nullptr && b->node_count > 0)
            GWNB_CUDA_TRY(cudaMemsetAsync(a->arrivals, 0, 2 * b->node_count * sizeof(std::uint32_t), s));
        GWNB_CUDA_TRY(cudaStreamSynchronize(s));
        if (host == k_err_stack_overflow)
            return set_error(GWNB_INTERNAL_ERROR, "query: traversal stack overflow (NaN written).");
        b->revision = 0;
        if (host & k_err_index)
            return set_error(GWNB_INTERNAL_ERROR, "bvh.refit: Bottom-up BVH refit did not converge.");
        return set_error(GWNB_INTERNAL_ERROR, "bvh: device status reported error bits " + std::to_string(host) + ".");
    }
    std::memcpy(&b->root.bounds, &rb, sizeof(rb));
    return GWNB_OK;
} catch (...) {
    return host_exception();
}

int gwnb_bvh4_refit_f32(const gwnb_geometry_f32 *g, gwnb_bvh4_f32 *b, gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::refit_bvh");
    GWNB_TRY(gwnb_bvh4_refit_async_f32(g, b, stream));
    return gwnb_bvh4_sync_status_f32(b, stream);
} catch (...) {
    return host_exception();
}

uint64_t gwnb_moment_node_bytes(int order) {
    if (order < 0 || order > 2)
        return 0;
    return static_cast<uint64_t>(moment_field_count(order)) * 16u;
}

static int moment_alloc(gwnb_bvh4_f32 const *b, int order, gwnb_moment4_f32 &m, cudaStream_t s) {
    m.order = order;
    m.node_count = b->node_count;
    if (b->node_count == 0)
        return GWNB_OK;
    auto *ma = new (std::nothrow) moment_aux_impl{};
    if (ma == nullptr)
        return set_error(GWNB_INTERNAL_ERROR, "out of host memory");
    m.aux = reinterpret_cast<gwnb_moment_aux *>(ma);
    std::uint64_t const nn = b->node_count;
    GWNB_TRY(alloc(reinterpret_cast<unsigned char **>(&m.nodes), nn * gwnb_moment_node_bytes(order), s));
    GWNB_TRY(alloc(&ma->qnodes, nn * 4 * qnode_f4_per_child(order), s));
    GWNB_TRY(alloc(&ma->qcounts, nn * 4, s));
    ma->payload_stride = moment_payload_bytes(order);
    GWNB_TRY(alloc(reinterpret_cast<unsigned char **>(&ma->payload), nn * ma->payload_stride, s));
    return GWNB_OK;
}

int gwnb_moment4_refit_f32(const gwnb_bvh4_f32 *b_in, int order, gwnb_moment4_f32 *out, gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::refit_moment");
    if (out == nullptr)
        return set_error(GWNB_INVALID_ARGUMENT, "bvh.refit.moment: output view is null.");
    if (order < 0 || order > 2)
        return set_error(GWNB_INVALID_ARGUMENT, "bvh.refit.moment: Taylor order must be 0, 1, or 2.");
    if (!bvh_valid(b_in))
        return set_error(GWNB_INVALID_ARGUMENT, "bvh.refit.moment: BVH accessor is invalid for moment refit.");
    cudaStream_t const s = as_cuda(stream);
    auto *b = const_cast<gwnb_bvh4_f32 *>(b_in);
    GWNB_TRY(ensure_bvh_aux(b, s));
    gwnb_moment4_f32 m{};
    int rc = moment_alloc(b, order, m, s);
    if (rc == GWNB_OK && b->node_count > 0)
        rc = refit_moments_async(b, &m, s);
    unsigned int host = 0;
    if (rc == GWNB_OK)
        rc = read_status(b, &host, s);
    if (rc == GWNB_OK && host != 0u) {
        auto *a = reinterpret_cast<bvh_aux_impl *>(b->aux);
        (void)cudaMemsetAsync(a->status, 0, sizeof(unsigned int), s);
        (void)cudaMemsetAsync(a->arrivals, 0, 2 * b->node_count * sizeof(std::uint32_t), s);
        rc = set_error(GWNB_INTERNAL_ERROR, "bvh.refit.moment: Bottom-up moment refit did not converge.");
    }
    if (rc != GWNB_OK) {
        free_moment(m, s);
        return rc;
    }
    m.bvh_revision = b->revision;
    *out = m;
    return GWNB_OK;
} catch (...) {
    return host_exception();
}

int gwnb_moment4_refit_async_f32(const gwnb_bvh4_f32 *b_in, gwnb_moment4_f32 *m, gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::refit_moment_async");
    if (m == nullptr || !bvh_valid(b_in))
        return set_error(GWNB_INVALID_ARGUMENT, "bvh.refit.moment: BVH accessor is invalid for moment refit.");
    if (m->node_count != b_in->node_count || (b_in->node_count > 0 && m->aux == nullptr))
        return set_error(GWNB_INVALID_ARGUMENT, "bvh.refit.moment: moment view does not match the BVH topology.");
    cudaStream_t const s = as_cuda(stream);
    auto *b = const_cast<gwnb_bvh4_f32 *>(b_in);
    GWNB_TRY(ensure_bvh_aux(b, s));
    if (b->node_count > 0)
        GWNB_TRY(refit_moments_async(b, m, s));
    m->bvh_revision = b->revision;
    return GWNB_OK;
} catch (...) {
    return host_exception();
}

void gwnb_moment4_release_f32(gwnb_moment4_f32 *m, gwnb_stream_t stream) {
    if (m != nullptr)
        free_moment(*m, as_cuda(stream));
}

// ---- queries ------------------------------------------------------------------------------------

static int check_query_spans(const float *qx, const float *qy, const float *qz, const float *out, uint64_t n) {
    if (!has_storage(qx, n) || !has_storage(qy, n) || !has_storage(qz, n) || !has_storage(out, n))
        return set_error(GWNB_INVALID_ARGUMENT, "Query/output spans must use non-null storage when non-empty.");
    return GWNB_OK;
}

int gwnb_winding_exact_batch_f32(const gwnb_bvh4_f32 *b, const float *qx, const float *qy, const float *qz,
                                 float *out, uint64_t n, int block_size, gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::query_exact");
    if (!bvh_valid(b))
        return set_error(GWNB_INVALID_ARGUMENT, "BVH object contains no queryable data.");
    if (block_size < 0 || block_size > 1024)
        return set_error(GWNB_INVALID_ARGUMENT, "Query batch block size must be in [1, 1024].");
    GWNB_TRY(check_query_spans(qx, qy, qz, out, n));
    if (n == 0)
        return GWNB_OK;
    return exact_batch(reinterpret_cast<triangle const *>(b->triangles), b->primitive_count, qx, qy, qz, out, n,
                       as_cuda(stream));
} catch (...) {
    return host_exception();
}

static int taylor_common(const gwnb_bvh4_f32 *b_in, const gwnb_moment4_f32 *m, const float *qx, const float *qy,
                         const float *qz, float *out, float *gx, float *gy, float *gz, uint32_t *sn, uint32_t *sf,
                         uint32_t *snear, uint64_t n, float beta, const gwnb_taylor_options *opt,
                         gwnb_stream_t stream, double *probe = nullptr) {
    if (!bvh_valid(b_in))
        return set_error(GWNB_INVALID_ARGUMENT, "BVH object contains no queryable data.");
    gwnb_taylor_options o{256, 64, 1, GWNB_NEAR_PLAIN, 1.0f / 16.0f};
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
    if (ref_internal(b_in->root.reference) && b_in->internal_stack_bound > static_cast<std::uint32_t>(o.stack_capacity))
        return set_error(GWNB_INVALID_ARGUMENT, "Traversal stack capacity is below the BVH internal stack bound.");
    if (ref_internal(b_in->root.reference) && b_in->internal_stack_bound > 128)
        return set_error(GWNB_INVALID_ARGUMENT, "Traversal stack bounds above 128 are not supported.");
    if (!moment_valid_for(m, b_in))
        return set_error(GWNB_INVALID_ARGUMENT, "Moment object is not aligned with the BVH.");
    if (!(beta >= 0.0f))
        return set_error(GWNB_INVALID_ARGUMENT, "Taylor accuracy scale must be nonnegative.");
    if (o.near_precision != GWNB_NEAR_PLAIN && o.near_precision != GWNB_NEAR_COMPENSATED)
        return set_error(GWNB_INVALID_ARGUMENT, "Unknown near-field precision mode.");
    if (o.per_thread < GWNB_WALK_WARP || o.per_thread > GWNB_WALK_TIMED)
        return set_error(GWNB_INVALID_ARGUMENT, "Unknown traversal (per_thread must be 0, 1 or 2).");
    if (!has_storage(qx, n) || !has_storage(qy, n) || !has_storage(qz, n))
        return set_error(GWNB_INVALID_ARGUMENT, "Query/output spans must use non-null storage when non-empty.");
    if (probe == nullptr && (out != nullptr || (gx == nullptr && sn == nullptr)))
        GWNB_TRY(check_query_spans(qx, qy, qz, out, n));
    if (n == 0)
        return GWNB_OK;
    if (n > 0xffffffffull)
        return set_error(GWNB_INVALID_ARGUMENT, "Query batch exceeds 2^32 - 1 queries.");
    cudaStream_t const s = as_cuda(stream);
    auto *b = const_cast<gwnb_bvh4_f32 *>(b_in);
    GWNB_TRY(ensure_bvh_aux(b, s));
    auto *a = reinterpret_cast<bvh_aux_impl *>(b->aux);
    auto *ma = reinterpret_cast<moment_aux_impl *>(m->aux);
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
    r.gx = gx;
    r.gy = gy;
    r.gz = gz;
    r.stat_nodes = sn;
    r.stat_far = sf;
    r.stat_near = snear;
    r.n = n;
    r.accuracy_scale = beta;
    r.block = o.block_size;
    r.stack_capacity = std::max<int>(static_cast<int>(b->internal_stack_bound), 1);
    r.sort_queries = o.sort_queries;
    r.near_mode = o.near_precision;
    r.per_thread = o.per_thread;
    r.fp64_threshold = o.fp64_threshold;
    r.fp64_count = a->fp64_count;
    r.status = a->status;
    r.probe = probe;
    if (o.near_precision == GWNB_NEAR_COMPENSATED && probe == nullptr)
        GWNB_CUDA_TRY(cudaMemsetAsync(a->fp64_count, 0, sizeof(unsigned long long), s));
    return taylor_batch(r, s);
}

int gwnb_winding_taylor_batch_f32(const gwnb_bvh4_f32 *b, const gwnb_moment4_f32 *m, const float *qx,
                                  const float *qy, const float *qz, float *out, uint64_t n, float beta,
                                  const gwnb_taylor_options *opt, gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::query_taylor");
    return taylor_common(b, m, qx, qy, qz, out, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, n, beta, opt,
                         stream);
} catch (...) {
    return host_exception();
}

int gwnb_winding_gradient_taylor_batch_f32(const gwnb_bvh4_f32 *b, const gwnb_moment4_f32 *m, const float *qx,
                                           const float *qy, const float *qz, float *gx, float *gy, float *gz,
                                           uint64_t n, float beta, const gwnb_taylor_options *opt,
                                           gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::query_taylor_gradient");
    if (n > 0 && (gx == nullptr || gy == nullptr || gz == nullptr))
        return set_error(GWNB_INVALID_ARGUMENT, "Query/output spans must use non-null storage when non-empty.");
    return taylor_common(b, m, qx, qy, qz, nullptr, gx, gy, gz, nullptr, nullptr, nullptr, n, beta, opt, stream);
} catch (...) {
    return host_exception();
}

int gwnb_winding_taylor_stats_f32(const gwnb_bvh4_f32 *b, const gwnb_moment4_f32 *m, const float *qx,
                                  const float *qy, const float *qz, uint64_t n, float beta, uint32_t *nodes,
                                  uint32_t *far_evals, uint32_t *near_tris, gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::query_taylor_stats");
    if (n > 0 && (nodes == nullptr || far_evals == nullptr || near_tris == nullptr))
        return set_error(GWNB_INVALID_ARGUMENT, "Statistics outputs must be non-null.");
    gwnb_taylor_options o{256, 0, 1, GWNB_NEAR_PLAIN, 1.0f / 16.0f};
    return taylor_common(b, m, qx, qy, qz, nullptr, nullptr, nullptr, nullptr, nodes, far_evals, near_tris, n, beta,
                         &o, stream);
} catch (...) {
    return host_exception();
}

int gwnb_taylor_form_probe_f32(const gwnb_bvh4_f32 *b, const gwnb_moment4_f32 *m, const float *qx, const float *qy,
                               const float *qz, uint64_t n, float beta, const gwnb_taylor_options *opt, double *out,
                               gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::taylor_form_probe");
    if (out == nullptr)
        return set_error(GWNB_INVALID_ARGUMENT, "taylor probe: output must be non-null.");
    for (int k = 0; k < 6; ++k)
        out[k] = 0.0;
    return taylor_common(b, m, qx, qy, qz, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, n, beta, opt,
                         stream, out);
} catch (...) {
    return host_exception();
}

int gwnb_winding_exact_geometry_fp64(const gwnb_geometry_f32 *g, const float *qx, const float *qy, const float *qz,
                                     double *out, uint64_t n, gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::query_exact_fp64");
    if (!geometry_valid(g))
        return set_error(GWNB_INVALID_ARGUMENT, "Geometry accessor is invalid.");
    if (!has_storage(qx, n) || !has_storage(qy, n) || !has_storage(qz, n) || !has_storage(out, n))
        return set_error(GWNB_INVALID_ARGUMENT, "Query/output spans must use non-null storage when non-empty.");
    return exact_batch_f64(*g, qx, qy, qz, out, n, as_cuda(stream));
} catch (...) {
    return host_exception();
}

int gwnb_query_order_f32(const gwnb_bvh4_f32 *b_in, const float *qx, const float *qy, const float *qz, uint64_t n,
                         uint32_t *order, gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::query_order");
    if (!bvh_valid(b_in))
        return set_error(GWNB_INVALID_ARGUMENT, "BVH object contains no queryable data.");
    if (!has_storage(qx, n) || !has_storage(qy, n) || !has_storage(qz, n) || !has_storage(order, n))
        return set_error(GWNB_INVALID_ARGUMENT, "Query/output spans must use non-null storage when non-empty.");
    cudaStream_t const s = as_cuda(stream);
    auto *b = const_cast<gwnb_bvh4_f32 *>(b_in);
    GWNB_TRY(ensure_bvh_aux(b, s));
    auto *a = reinterpret_cast<bvh_aux_impl *>(b->aux);
    return query_order(a->root_bounds, qx, qy, qz, n, order, s, a->status);
} catch (...) {
    return host_exception();
}

int gwnb_bvh4_fp64_fallback_count(const gwnb_bvh4_f32 *b, uint64_t *count, gwnb_stream_t stream) try {
    if (b == nullptr || b->aux == nullptr || count == nullptr)
        return set_error(GWNB_INVALID_ARGUMENT, "fp64 counter: BVH has no device state.");
    auto *a = reinterpret_cast<bvh_aux_impl *>(b->aux);
    unsigned long long host = 0;
    cudaStream_t const s = as_cuda(stream);
    GWNB_CUDA_TRY(cudaMemcpyAsync(&host, a->fp64_count, sizeof(host), cudaMemcpyDeviceToHost, s));
    GWNB_CUDA_TRY(cudaStreamSynchronize(s));
    *count = host;
    return GWNB_OK;
} catch (...) {
    return host_exception();
}

int gwnb_winding_taylor_forward_f32(const gwnb_bvh4_f32 *b, const gwnb_moment4_f32 *m, const float *qx,
                                    const float *qy, const float *qz, float *out, uint64_t n, float beta,
                                    const gwnb_taylor_options *opt, gwnb_taylor_saved_f32 *saved,
                                    gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::taylor_forward");
    if (saved == nullptr)
        return set_error(GWNB_INVALID_ARGUMENT, "Taylor forward: saved state must be non-null.");
    if (m == nullptr || (m->order != 0 && m->order != 1))
        return set_error(GWNB_INVALID_ARGUMENT, "The Taylor adjoint supports orders 0 and 1.");
    GWNB_TRY(taylor_common(b, m, qx, qy, qz, out, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, n, beta, opt,
                           stream));
    gwnb_taylor_options o{256, 64, 1, GWNB_NEAR_PLAIN, 1.0f / 16.0f, 0};
    if (opt != nullptr)
        o = *opt;
    if (o.block_size == 0)
        o.block_size = 256;
    if (o.stack_capacity == 0)
        o.stack_capacity = 64;
    saved->query_x = qx;
    saved->query_y = qy;
    saved->query_z = qz;
    saved->count = n;
    saved->accuracy_scale = beta;
    saved->order = m->order;
    saved->bvh_revision = b->revision;
    saved->options = o;
    return GWNB_OK;
} catch (...) {
    return host_exception();
}

int gwnb_winding_taylor_backward_f32(const gwnb_taylor_saved_f32 *saved, const gwnb_geometry_f32 *g,
                                     const gwnb_bvh4_f32 *b_in, const gwnb_moment4_f32 *m, const float *gout,
                                     float *dvx, float *dvy, float *dvz, float *dqx, float *dqy, float *dqz,
                                     gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::taylor_backward");
    if (saved == nullptr)
        return set_error(GWNB_INVALID_ARGUMENT, "Taylor backward: saved state must be non-null.");
    if (saved->order != 0 && saved->order != 1)
        return set_error(GWNB_INVALID_ARGUMENT, "The Taylor adjoint supports orders 0 and 1.");
    if (!bvh_valid(b_in))
        return set_error(GWNB_INVALID_ARGUMENT, "BVH object contains no queryable data.");
    if (b_in->revision != saved->bvh_revision)
        return set_error(GWNB_INVALID_ARGUMENT, "Taylor backward: the BVH changed since the forward pass.");
    if (!moment_valid_for(m, b_in) || m->order != saved->order)
        return set_error(GWNB_INVALID_ARGUMENT, "Moment object is not aligned with the BVH.");
    bool const want_v = dvx != nullptr || dvy != nullptr || dvz != nullptr;
    bool const want_q = dqx != nullptr || dqy != nullptr || dqz != nullptr;
    if (want_v && (dvx == nullptr || dvy == nullptr || dvz == nullptr))
        return set_error(GWNB_INVALID_ARGUMENT, "Vertex gradient outputs must be all null or all non-null.");
    if (want_q && (dqx == nullptr || dqy == nullptr || dqz == nullptr))
        return set_error(GWNB_INVALID_ARGUMENT, "Query gradient outputs must be all null or all non-null.");
    if (want_v) {
        if (!geometry_valid(g))
            return set_error(GWNB_INVALID_ARGUMENT, "Geometry accessor is invalid.");
        if (g->triangle_count != b_in->primitive_count)
            return set_error(GWNB_INVALID_ARGUMENT, "Taylor backward: geometry does not match the BVH.");
    }
    std::uint64_t const n = saved->count;
    if (!has_storage(gout, n) || !has_storage(saved->query_x, n) || !has_storage(saved->query_y, n) ||
        !has_storage(saved->query_z, n))
        return set_error(GWNB_INVALID_ARGUMENT, "Query/output spans must use non-null storage when non-empty.");
    if (ref_internal(b_in->root.reference) && b_in->internal_stack_bound > 64)
        return set_error(GWNB_INVALID_ARGUMENT, "Taylor backward: stack bounds above 64 are not supported.");
    if (!want_v && !want_q)
        return GWNB_OK;
    cudaStream_t const s = as_cuda(stream);
    auto *b = const_cast<gwnb_bvh4_f32 *>(b_in);
    GWNB_TRY(ensure_bvh_aux(b, s));
    auto *a = reinterpret_cast<bvh_aux_impl *>(b->aux);
    auto *ma = reinterpret_cast<moment_aux_impl *>(m->aux);
    adjoint_request r{};
    r.order = saved->order;
    r.qnodes = ma != nullptr ? ma->qnodes : nullptr;
    r.qcounts = ma != nullptr ? ma->qcounts : nullptr;
    r.tri48 = a->tri48;
    r.triangles = reinterpret_cast<triangle const *>(b->triangles);
    r.nodes = reinterpret_cast<node4 const *>(b->nodes);
    r.primitive_count = b->primitive_count;
    r.node_count = b->node_count;
    r.root_ref = b->root.reference;
    r.root_bounds = a->root_bounds;
    r.parent_slot = a->parent_slot;
    r.primitive_indices = b->primitive_indices;
    r.payload = ma != nullptr ? static_cast<float const *>(ma->payload) : nullptr;
    r.payload_floats = ma != nullptr ? ma->payload_stride / sizeof(float) : 0;
    if (want_v)
        r.g = *g;
    r.qx = saved->query_x;
    r.qy = saved->query_y;
    r.qz = saved->query_z;
    r.grad_out = gout;
    r.dvx = want_v ? dvx : nullptr;
    r.dvy = want_v ? dvy : nullptr;
    r.dvz = want_v ? dvz : nullptr;
    r.dqx = want_q ? dqx : nullptr;
    r.dqy = want_q ? dqy : nullptr;
    r.dqz = want_q ? dqz : nullptr;
    r.n = n;
    r.accuracy_scale = saved->accuracy_scale;
    r.block = 256; // the backward traversal's own launch shape (its kernels are bounded to 256 threads)
    r.stack_capacity = std::max<int>(static_cast<int>(b->internal_stack_bound), 1);
    r.sort_queries = saved->options.sort_queries;
    r.status = a->status;
    return taylor_adjoint(r, s);
} catch (...) {
    return host_exception();
}

} // extern "C"
