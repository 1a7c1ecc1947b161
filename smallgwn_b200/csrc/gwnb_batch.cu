// Batched dynamic meshes: many BVHs refit and queried per frame in three persistent launches.
//
// smallgwn serves one mesh per call, and every refit synchronizes with the host
// (detail/gwn_bvh_refit_impl.cuh:324, detail/gwn_bvh_refit_moment_impl.cuh:260). Here a batch holds
// the device descriptors of all its meshes: a frame is the batched bounds refit (one work item per
// leaf-bearing node of every BVH), the batched moment refit, and one traversal launch over every
// mesh's queries (warp-aligned ranges of a common slot space). Nothing in a frame allocates or
// synchronizes, so applications capture frames (with their own vertex updates) in a CUDA graph.
//
// The autotuner times candidate launch shapes -- refit block size; query block size, traversal
// form (a warp of 32 Hilbert-adjacent queries walking one traversal, or one traversal per thread),
// Hilbert-ordered or input order, persistent grid size -- on the batch itself and keeps the fastest.
//
// Refitting keeps the topology built for the rest shape; as the meshes deform, the boxes of a
// refit tree grow and overlap and every query visits more nodes. The batch measures each tree's
// quality as its surface-area cost (the sum over nodes of the children's box half-areas, over the
// root's half-area: the expected number of child boxes a uniformly placed probe enters) relative to
// the cost when the tree was built, and rebuilds the trees whose cost grew past a caller's
// threshold (gwnb_batch_rebuild_f32), between frames.
#include "gwnb_internal.cuh"

#include <algorithm>
#include <cstdio>
#include <new>
#include <string>
#include <vector>

// The arrays a mesh's BVH and moment objects held when the batch derived its descriptors from them.
struct gwnb_batch_ident {
    void const *bvh_nodes;
    void const *bvh_aux;
    void const *moment_nodes;
    void const *moment_aux;
};

struct gwnb_batch {
    std::vector<gwnb_batch_mesh_f32> meshes; // the caller's mesh descriptors (objects updated in place)
    std::vector<gwnb_batch_ident> idents;    // per mesh, the arrays the device descriptors point into
    std::vector<double> base_cost;           // surface-area cost of each tree when built
    float beta = 2.0f;
    gwnb_taylor_options options{};
    int order = 0;
    std::vector<gwnb_bvh4_f32 *> bvhs;
    std::vector<unsigned int *> status_words;
    gwnb::batch_refit_state refit{};
    gwnb::batch_query_state query{};
    gwnb_batch_tuning tuning{128, 256, 0, 1, 8, 0.0f};
    unsigned int **d_status = nullptr; // device copy of status_words
    unsigned int *d_flags = nullptr;   // OR of every mesh's status word
    cudaStream_t stream = nullptr;     // stream the batch's arrays were allocated on
    bool ready = false;                // the device descriptors are complete (prepare_states succeeded)
};

namespace gwnb {
namespace {

__global__ void k_gather_status(unsigned int *const *__restrict__ words, std::uint32_t n, unsigned int *out) {
    unsigned int v = 0;
    for (std::uint32_t i = threadIdx.x; i < n; i += blockDim.x)
        v |= *words[i];
    if (v != 0u)
        atomicOr(out, v);
}

void release_batch(gwnb_batch *b, cudaStream_t s) {
    batch_refit_release(b->refit, s);
    batch_query_release(b->query, s);
    release(b->d_status, s);
    release(b->d_flags, s);
}

// Surface-area cost terms of one tree: out[0] += sum over nodes of the children's box half-areas,
// out[1] = the half-area of the union of the root node's children (the root box).
__global__ void __launch_bounds__(256)
    k_tree_cost(node4 const *__restrict__ nodes, std::uint64_t node_count, double *out) {
    std::uint64_t const n = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    double sum = 0.0;
    if (n < node_count) {
        aabb u{__int_as_float(0x7f800000), __int_as_float(0x7f800000), __int_as_float(0x7f800000),
               -__int_as_float(0x7f800000), -__int_as_float(0x7f800000), -__int_as_float(0x7f800000)};
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            if (!ref_valid(nodes[n].c[c].reference))
                continue;
            aabb const &b = nodes[n].c[c].bounds;
            sum += static_cast<double>(aabb_half_area(b));
            u = aabb_union(u, b);
        }
        if (n == 0)
            out[1] = static_cast<double>(aabb_half_area(u));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if ((threadIdx.x & 31u) == 0u && sum != 0.0)
        atomicAdd(out, sum);
}

// Each mesh's surface-area cost (1 for a tree whose root is a leaf). Synchronizes the stream.
int tree_costs(gwnb_batch *b, std::vector<double> &cost, cudaStream_t s) {
    std::size_t const m = b->meshes.size();
    double *d = nullptr;
    GWNB_TRY(alloc(&d, 2 * m, s));
    int rc = GWNB_OK;
    if (cudaMemsetAsync(d, 0, 2 * m * sizeof(double), s) != cudaSuccess)
        rc = set_cuda_error(cudaGetLastError(), "batch tree cost");
    for (std::size_t i = 0; i < m && rc == GWNB_OK; ++i) {
        gwnb_bvh4_f32 const *bv = b->meshes[i].bvh;
        if (bv->node_count == 0)
            continue;
        note_launch(), k_tree_cost<<<static_cast<unsigned>((bv->node_count + 255) / 256), 256, 0, s>>>(
            reinterpret_cast<node4 const *>(bv->nodes), bv->node_count, d + 2 * i);
        if (cudaGetLastError() != cudaSuccess)
            rc = set_cuda_error(cudaGetLastError(), "batch tree cost");
    }
    std::vector<double> h(2 * m, 0.0);
    if (rc == GWNB_OK && (cudaMemcpyAsync(h.data(), d, 2 * m * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                          cudaStreamSynchronize(s) != cudaSuccess))
        rc = set_cuda_error(cudaGetLastError(), "batch tree cost read-back");
    release(d, s);
    if (rc != GWNB_OK)
        return rc;
    cost.assign(m, 1.0);
    for (std::size_t i = 0; i < m; ++i)
        if (b->meshes[i].bvh->node_count > 0 && h[2 * i + 1] > 0.0)
            cost[i] = h[2 * i] / h[2 * i + 1];
    return GWNB_OK;
}

// The batch's device descriptors (refit items, traversal descriptors and Hilbert orders, status
// words) from its meshes' current objects; replaces any previous ones.
int prepare_states_impl(gwnb_batch *b, cudaStream_t s) {
    batch_refit_release(b->refit, s);
    batch_query_release(b->query, s);
    b->refit = batch_refit_state{};
    b->query = batch_query_state{};
    std::uint32_t const mesh_count = static_cast<std::uint32_t>(b->meshes.size());
    std::vector<gwnb_geometry_f32> geoms(mesh_count);
    std::vector<gwnb_moment4_f32 *> moms(mesh_count);
    std::vector<taylor_request> reqs(mesh_count);
    b->bvhs.resize(mesh_count);
    b->status_words.resize(mesh_count);
    for (uint32_t i = 0; i < mesh_count; ++i) {
        gwnb_batch_mesh_f32 const &m = b->meshes[i];
        GWNB_TRY(ensure_bvh_aux(m.bvh, s));
        auto *a = reinterpret_cast<bvh_aux_impl *>(m.bvh->aux);
        auto *ma = reinterpret_cast<moment_aux_impl *>(m.moment->aux);
        geoms[i] = m.geometry;
        moms[i] = m.moment;
        b->bvhs[i] = m.bvh;
        b->status_words[i] = a->status;
        taylor_request &r = reqs[i];
        r.order = b->order;
        r.qnodes = ma != nullptr ? ma->qnodes : nullptr;
        r.qcounts = ma != nullptr ? ma->qcounts : nullptr;
        r.tri48 = a->tri48;
        r.primitive_count = m.bvh->primitive_count;
        r.node_count = m.bvh->node_count;
        r.root_ref = m.bvh->root.reference;
        r.root_bounds = a->root_bounds;
        r.qx = m.query_x;
        r.qy = m.query_y;
        r.qz = m.query_z;
        r.out = m.output;
        r.n = m.query_count;
        r.accuracy_scale = b->beta;
        r.stack_capacity = std::max<int>(static_cast<int>(m.bvh->internal_stack_bound), 1);
        r.sort_queries = 1;
        r.near_mode = b->options.near_precision;
        r.fp64_threshold = b->options.fp64_threshold;
        r.fp64_count = a->fp64_count;
        r.status = a->status;
    }
    b->idents.resize(mesh_count);
    for (uint32_t i = 0; i < mesh_count; ++i)
        b->idents[i] = gwnb_batch_ident{b->meshes[i].bvh->nodes, b->meshes[i].bvh->aux, b->meshes[i].moment->nodes,
                                        b->meshes[i].moment->aux};
    GWNB_TRY(batch_refit_prepare(geoms.data(), b->bvhs.data(), moms.data(), mesh_count, b->order, &b->refit, s));
    GWNB_TRY(batch_query_prepare(reqs.data(), mesh_count, &b->query, s));
    if (b->d_status == nullptr)
        GWNB_TRY(alloc(&b->d_status, mesh_count, s));
    if (b->d_flags == nullptr)
        GWNB_TRY(alloc(&b->d_flags, 1, s));
    if (cudaMemcpyAsync(b->d_status, b->status_words.data(), mesh_count * sizeof(unsigned int *),
                        cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return set_cuda_error(cudaGetLastError(), "batch descriptors");
    return GWNB_OK;
}

// The batch's device descriptors point into its meshes' BVH and moment arrays as they were when
// it derived them. A BVH built again or moments refit into new arrays outside the batch (the caller
// replacing an object it lent) leave those pointers dangling: every entry point that launches over
// or reads the meshes refuses the batch from then on.
int check_current(gwnb_batch const *b) {
    for (std::size_t i = 0; i < b->meshes.size(); ++i) {
        gwnb_batch_mesh_f32 const &m = b->meshes[i];
        gwnb_batch_ident const &id = b->idents[i];
        if (m.bvh->nodes != id.bvh_nodes || m.bvh->aux != id.bvh_aux || m.moment->nodes != id.moment_nodes ||
            m.moment->aux != id.moment_aux)
            return set_error(GWNB_INVALID_ARGUMENT,
                             "batch: mesh " + std::to_string(i) + "'s BVH or moments were replaced after the batch "
                             "was made (a build or moment refit outside the batch); make a new batch.");
    }
    return GWNB_OK;
}

// prepare_states_impl with the batch marked ready only when every descriptor is in place; on a
// failure the partial descriptors are released and the frame entry points refuse the batch.
int prepare_states(gwnb_batch *b, cudaStream_t s) {
    b->ready = false;
    int const rc = prepare_states_impl(b, s);
    if (rc != GWNB_OK) {
        batch_refit_release(b->refit, s);
        batch_query_release(b->query, s);
        b->refit = batch_refit_state{};
        b->query = batch_query_state{};
        return rc;
    }
    b->ready = true;
    return GWNB_OK;
}

int run_stages(gwnb_batch *b, gwnb_batch_tuning const &t, unsigned stages, cudaStream_t s) {
    if (!b->ready)
        return set_error(GWNB_INTERNAL_ERROR, "batch: its device descriptors are incomplete after a failed rebuild; "
                                              "call rebuild again or release the batch.");
    GWNB_TRY(check_current(b));
    bool const bounds = (stages & GWNB_BATCH_REFIT) != 0u, moments = (stages & GWNB_BATCH_MOMENTS) != 0u;
    if (bounds || moments)
        GWNB_TRY(batch_refit_launch(b->refit, t.refit_block, bounds, moments, s));
    if ((stages & GWNB_BATCH_QUERY) != 0u) {
        batch_query_config const c{t.query_block, t.per_thread, t.sorted, t.grid_scale};
        return batch_query_launch(b->query, c, s);
    }
    return GWNB_OK;
}

int frame(gwnb_batch *b, gwnb_batch_tuning const &t, cudaStream_t s) {
    return run_stages(b, t, GWNB_BATCH_REFIT | GWNB_BATCH_MOMENTS | GWNB_BATCH_QUERY, s);
}

bool tuning_valid(gwnb_batch_tuning const &t) {
    return t.refit_block >= 32 && t.refit_block <= 256 && (t.refit_block % 32) == 0 && t.query_block >= 32 &&
           t.query_block <= 256 && (t.query_block % 32) == 0 && (t.per_thread == 0 || t.per_thread == 1) &&
           (t.sorted == 0 || t.sorted == 1) && t.grid_scale >= 1 && t.grid_scale <= 64;
}

} // namespace
} // namespace gwnb

using namespace gwnb;

extern "C" {

int gwnb_batch_create_f32(const gwnb_batch_mesh_f32 *meshes, uint32_t mesh_count, float beta,
                          const gwnb_taylor_options *opt, gwnb_batch **out, gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::batch.create");
    if (out == nullptr)
        return set_error(GWNB_INVALID_ARGUMENT, "batch: output handle must be non-null.");
    *out = nullptr;
    if (mesh_count == 0 || meshes == nullptr)
        return set_error(GWNB_INVALID_ARGUMENT, "batch: at least one mesh is required.");
    if (!(beta >= 0.0f))
        return set_error(GWNB_INVALID_ARGUMENT, "Taylor accuracy scale must be nonnegative.");
    gwnb_taylor_options o{256, 64, 1, GWNB_NEAR_PLAIN, 1.0f / 16.0f, 0};
    if (opt != nullptr)
        o = *opt;
    if (o.near_precision != GWNB_NEAR_PLAIN && o.near_precision != GWNB_NEAR_COMPENSATED)
        return set_error(GWNB_INVALID_ARGUMENT, "Unknown near-field precision mode.");
    int const order = meshes[0].moment != nullptr ? meshes[0].moment->order : -1;
    for (uint32_t i = 0; i < mesh_count; ++i) {
        gwnb_batch_mesh_f32 const &m = meshes[i];
        if (!geometry_valid(&m.geometry))
            return set_error(GWNB_INVALID_ARGUMENT, "batch: mesh " + std::to_string(i) + " has an invalid geometry.");
        if (!bvh_valid(m.bvh))
            return set_error(GWNB_INVALID_ARGUMENT, "batch: mesh " + std::to_string(i) + " has no queryable BVH.");
        if (m.geometry.triangle_count != m.bvh->primitive_count)
            return set_error(GWNB_INVALID_ARGUMENT,
                             "batch: mesh " + std::to_string(i) + " geometry does not match its BVH.");
        if (!moment_valid_for(m.moment, m.bvh) || m.moment->order != order)
            return set_error(GWNB_INVALID_ARGUMENT,
                             "batch: mesh " + std::to_string(i) + " moments are stale or of another order.");
        if (!has_storage(m.query_x, m.query_count) || !has_storage(m.query_y, m.query_count) ||
            !has_storage(m.query_z, m.query_count) || !has_storage(m.output, m.query_count))
            return set_error(GWNB_INVALID_ARGUMENT,
                             "batch: mesh " + std::to_string(i) + " query/output spans must be non-null.");
        if (m.query_count > 0xffffffffull)
            return set_error(GWNB_INVALID_ARGUMENT, "Query batch exceeds 2^32 - 1 queries.");
        if (ref_internal(m.bvh->root.reference) && m.bvh->internal_stack_bound > 64)
            return set_error(GWNB_INVALID_ARGUMENT, "Batched traversal supports stack bounds up to 64.");
    }
    cudaStream_t const s = as_cuda(stream);
    auto *b = new (std::nothrow) gwnb_batch{};
    if (b == nullptr)
        return set_error(GWNB_INTERNAL_ERROR, "out of host memory");
    b->stream = s;
    b->meshes.assign(meshes, meshes + mesh_count);
    b->beta = beta;
    b->options = o;
    b->order = order;
    int rc = prepare_states(b, s);
    if (rc == GWNB_OK)
        rc = tree_costs(b, b->base_cost, s);
    if (rc != GWNB_OK) {
        release_batch(b, s);
        delete b;
        return rc;
    }
    *out = b;
    return GWNB_OK;
} catch (...) {
    return host_exception();
}

int gwnb_batch_quality_f32(gwnb_batch *b, float *cost_ratio, gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::batch.quality");
    if (b == nullptr || cost_ratio == nullptr)
        return set_error(GWNB_INVALID_ARGUMENT, "batch: null handle or output.");
    GWNB_TRY(check_current(b));
    std::vector<double> cost;
    GWNB_TRY(tree_costs(b, cost, as_cuda(stream)));
    for (std::size_t i = 0; i < cost.size(); ++i)
        cost_ratio[i] = static_cast<float>(b->base_cost[i] > 0.0 ? cost[i] / b->base_cost[i] : 1.0);
    return GWNB_OK;
} catch (...) {
    return host_exception();
}

int gwnb_batch_rebuild_f32(gwnb_batch *b, float threshold, int method, uint32_t radius, uint32_t *rebuilt,
                           gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::batch.rebuild");
    if (b == nullptr)
        return set_error(GWNB_INVALID_ARGUMENT, "batch: null handle.");
    if (!(threshold >= 1.0f))
        return set_error(GWNB_INVALID_ARGUMENT, "batch: the rebuild threshold is a cost ratio of at least 1.");
    GWNB_TRY(check_current(b));
    cudaStream_t const s = as_cuda(stream);
    std::vector<double> cost;
    GWNB_TRY(tree_costs(b, cost, s));
    std::uint32_t count = 0;
    std::vector<char> redo(b->meshes.size(), 0);
    int rc = GWNB_OK;
    for (std::size_t i = 0; i < b->meshes.size() && rc == GWNB_OK; ++i) {
        if (!(cost[i] > threshold * b->base_cost[i]))
            continue;
        gwnb_batch_mesh_f32 &m = b->meshes[i];
        // both new objects first: on failure the mesh keeps its current BVH and moments
        gwnb_bvh4_f32 fresh{};
        if ((rc = gwnb_bvh4_build_f32(&m.geometry, method, radius, 64, &fresh, stream)) != GWNB_OK)
            break;
        gwnb_moment4_f32 mom{};
        if ((rc = gwnb_moment4_refit_f32(&fresh, b->order, &mom, stream)) != GWNB_OK) {
            gwnb_bvh4_release_f32(&fresh, stream);
            break;
        }
        gwnb_bvh4_release_f32(m.bvh, stream);
        *m.bvh = fresh;
        gwnb_moment4_release_f32(m.moment, stream);
        *m.moment = mom;
        redo[i] = 1;
        ++count;
    }
    if (count > 0 || !b->ready) {
        // the descriptors follow the replaced objects even when a later mesh failed (and are
        // prepared again after an earlier rebuild could not finish them)
        int const prc = prepare_states(b, s);
        if (rc == GWNB_OK)
            rc = prc;
    }
    if (rc != GWNB_OK)
        return rc;
    if (count > 0) {
        GWNB_TRY(tree_costs(b, cost, s));
        for (std::size_t i = 0; i < cost.size(); ++i)
            if (redo[i])
                b->base_cost[i] = cost[i]; // the other trees keep the cost they were built with
    }
    if (rebuilt != nullptr)
        *rebuilt = count;
    return GWNB_OK;
} catch (...) {
    return host_exception();
}

int gwnb_batch_set_tuning_f32(gwnb_batch *b, const gwnb_batch_tuning *t) try {
    if (b == nullptr || t == nullptr || !tuning_valid(*t))
        return set_error(GWNB_INVALID_ARGUMENT, "batch: invalid tuning.");
    b->tuning = *t;
    return GWNB_OK;
} catch (...) {
    return host_exception();
}

int gwnb_batch_frame_f32(gwnb_batch *b, gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::batch.frame");
    if (b == nullptr)
        return set_error(GWNB_INVALID_ARGUMENT, "batch: null handle.");
    return frame(b, b->tuning, as_cuda(stream));
} catch (...) {
    return host_exception();
}

int gwnb_batch_run_f32(gwnb_batch *b, unsigned int stages, gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::batch.run");
    if (b == nullptr)
        return set_error(GWNB_INVALID_ARGUMENT, "batch: null handle.");
    if ((stages & ~(GWNB_BATCH_REFIT | GWNB_BATCH_MOMENTS | GWNB_BATCH_QUERY)) != 0u)
        return set_error(GWNB_INVALID_ARGUMENT, "batch: unknown stage bits.");
    return run_stages(b, b->tuning, stages, as_cuda(stream));
} catch (...) {
    return host_exception();
}

int gwnb_batch_tune_f32(gwnb_batch *b, int reps, gwnb_batch_tuning *chosen, gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::batch.tune");
    if (b == nullptr || reps <= 0)
        return set_error(GWNB_INVALID_ARGUMENT, "batch: tuning needs a handle and a positive repetition count.");
    cudaStream_t const s = as_cuda(stream);
    std::vector<gwnb_batch_tuning> cand;
    for (int refit_block : {128, 256})
        for (int per_thread : {0, 1})
            for (int sorted : {1, 0})
                for (int block : {128, 256})
                    for (int scale : {4, 8, 16})
                        cand.push_back(gwnb_batch_tuning{refit_block, block, per_thread, sorted, scale, 0.0f});
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    GWNB_CUDA_TRY(cudaEventCreate(&e0));
    GWNB_CUDA_TRY(cudaEventCreate(&e1));
    int rc = GWNB_OK;
    gwnb_batch_tuning best{};
    float best_ms = -1.0f;
    for (gwnb_batch_tuning &t : cand) {
        if ((rc = frame(b, t, s)) != GWNB_OK) // warm-up (and one-time attribute setup)
            break;
        if (cudaEventRecord(e0, s) != cudaSuccess) {
            rc = set_cuda_error(cudaGetLastError(), "batch tuning");
            break;
        }
        for (int r = 0; r < reps && rc == GWNB_OK; ++r)
            rc = frame(b, t, s);
        if (rc != GWNB_OK)
            break;
        float ms = 0.0f;
        if (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
            cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
            rc = set_cuda_error(cudaGetLastError(), "batch tuning");
            break;
        }
        t.frame_ms = ms / static_cast<float>(reps);
        if (best_ms < 0.0f || t.frame_ms < best_ms) {
            best_ms = t.frame_ms;
            best = t;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != GWNB_OK)
        return rc;
    b->tuning = best;
    // leave the chosen shape's one-time setup done, so the next frame can be captured
    GWNB_TRY(frame(b, best, s));
    GWNB_CUDA_TRY(cudaStreamSynchronize(s));
    if (chosen != nullptr)
        *chosen = best;
    return GWNB_OK;
} catch (...) {
    return host_exception();
}

int gwnb_batch_sync_f32(gwnb_batch *b, gwnb_stream_t stream) try {
    if (b == nullptr)
        return set_error(GWNB_INVALID_ARGUMENT, "batch: null handle.");
    if (!b->ready) // the device copy of the status words may still name the replaced objects
        return set_error(GWNB_INTERNAL_ERROR, "batch: its device descriptors are incomplete after a failed rebuild; "
                                              "call rebuild again or release the batch.");
    GWNB_TRY(check_current(b));
    cudaStream_t const s = as_cuda(stream);
    GWNB_CUDA_TRY(cudaMemsetAsync(b->d_flags, 0, sizeof(unsigned int), s));
    note_launch(), k_gather_status<<<1, 256, 0, s>>>(b->d_status, static_cast<std::uint32_t>(b->status_words.size()), b->d_flags);
    GWNB_CUDA_TRY(cudaGetLastError());
    unsigned int flags = 0;
    GWNB_CUDA_TRY(cudaMemcpyAsync(&flags, b->d_flags, sizeof(flags), cudaMemcpyDeviceToHost, s));
    GWNB_CUDA_TRY(cudaStreamSynchronize(s));
    if (flags != 0u)
        return set_error(GWNB_INTERNAL_ERROR, "batch: device error bits 0x" + [&] {
            char buf[16];
            std::snprintf(buf, sizeof(buf), "%x", flags);
            return std::string(buf);
        }() + " (index, topology, wait timeout, stack overflow) on at least one mesh.");
    return GWNB_OK;
} catch (...) {
    return host_exception();
}

int gwnb_batch_release_f32(gwnb_batch *b, gwnb_stream_t stream) try {
    if (b == nullptr)
        return GWNB_OK;
    cudaStream_t const s = stream != nullptr ? as_cuda(stream) : b->stream;
    release_batch(b, s);
    delete b;
    return GWNB_OK;
} catch (...) {
    return host_exception();
}

} // extern "C"
