/*
 * gwnb.h -- C ABI of the B200-native generalized-winding-number library (libgwnb.so).
 *
 * Every entry point takes plain pointers, sizes and a CUDA stream, and returns an int status code
 * (GWNB_OK, GWNB_INVALID_ARGUMENT, GWNB_CUDA_RUNTIME_ERROR, GWNB_INTERNAL_ERROR). The message for
 * the last failure on the calling host thread is returned by gwnb_last_error_message().
 *
 * The entry points replace the public C++ template API of smallgwn (namespace gwn, headers under
 * include/gwn/ of that project); the citation beside each declaration names the interface it
 * replaces. The C++ drop-in headers in include/gwn/ of this repository are thin inline wrappers
 * over these symbols, so existing smallgwn callers keep their source code.
 *
 * Supported instantiation: Width = 4, Real = float, Index = uint32_t, MortonCode in {uint32_t,
 * uint64_t}, Taylor Order in {0, 1, 2}.
 *
 * Memory layouts that cross this boundary are identical to smallgwn's:
 *   - gwnb_child_f32        == gwn::gwn_bvh_child<float>      (32 B, include/gwn/gwn_bvh.cuh:55-103)
 *   - gwnb_node4_f32        == gwn::gwn_bvh_node<4, float>    (128 B, :108-124)
 *   - gwnb_triangle_f32     == gwn::gwn_bvh_triangle<float>   (36 B, :39-49)
 *   - moment nodes          == gwn::gwn_bvh_moment_node<4, Order, float> field-SoA (:144-202)
 * Objects own device memory allocated with cudaMallocAsync on the stream passed to the call that
 * created them; gwnb_*_release frees it with cudaFreeAsync on the stream given to the release.
 */
#ifndef GWNB_H
#define GWNB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define GWNB_API __attribute__((visibility("default")))
#else
#define GWNB_API
#endif

/* cudaStream_t without pulling in the CUDA headers. */
typedef struct CUstream_st *gwnb_stream_t;

enum {
    GWNB_OK = 0,
    GWNB_INVALID_ARGUMENT = 1,
    GWNB_CUDA_RUNTIME_ERROR = 2,
    GWNB_INTERNAL_ERROR = 3,
};

enum { GWNB_METHOD_HPLOC = 0, GWNB_METHOD_LBVH = 1 };

/* Precision of the exact near-field solid angle inside the Taylor traversal. */
enum {
    GWNB_NEAR_PLAIN = 0,       /* FP32 Van Oosterom-Strackee, as smallgwn evaluates it        */
    GWNB_NEAR_COMPENSATED = 1, /* two-product compensated FP32, FP64 on flagged triangles    */
};

/* Walk of the Taylor traversal (gwnb_taylor_options::per_thread). Both walks give identical results.
 * GWNB_WALK_TIMED: the first call of a kind (moment object, order, precision, gradient or value,
 * accuracy scale, ordered or not, device, floor(log2 n)) walks warp-cooperatively and the second per
 * thread, each timed with CUDA events; once both timings have completed, calls of that kind take the
 * faster walk (until then the warp walk). Nothing blocks on the timings; calls under stream capture
 * record nothing and take the decided walk, else the warp walk. */
enum {
    GWNB_WALK_WARP = 0,   /* 32 ordered queries per warp walk one traversal together (default) */
    GWNB_WALK_THREAD = 1, /* one independent traversal per query                               */
    GWNB_WALK_TIMED = 2,  /* the faster of the two, chosen from timed calls of the same kind    */
};

typedef struct gwnb_aabb_f32 {
    float min_x, min_y, min_z, max_x, max_y, max_z;
} gwnb_aabb_f32;

typedef struct gwnb_child_f32 {
    gwnb_aabb_f32 bounds;
    uint64_t reference; /* bits 0-46 offset, bit 47 valid, bits 48-63 primitive count */
} gwnb_child_f32;

typedef struct gwnb_node4_f32 {
    gwnb_child_f32 children[4];
} gwnb_node4_f32;

typedef struct gwnb_triangle_f32 {
    float v0_x, v0_y, v0_z, e1_x, e1_y, e1_z, e2_x, e2_y, e2_z;
} gwnb_triangle_f32;

/* Device geometry view; mirrors gwn::gwn_geometry_accessor<float, uint32_t>
 * (include/gwn/gwn_geometry.cuh:19-49). */
typedef struct gwnb_geometry_f32 {
    float *vertex_x, *vertex_y, *vertex_z;
    uint64_t vertex_count;
    uint32_t *tri_i0, *tri_i1, *tri_i2;
    uint64_t triangle_count;
} gwnb_geometry_f32;

/* Library-owned derived state of a BVH (parent links, arrival counters, padded triangle records,
 * device error word). Opaque to callers. */
typedef struct gwnb_bvh_aux gwnb_bvh_aux;

/* Device BVH view; field meaning mirrors gwn::gwn_bvh_accessor<4, float, uint32_t>
 * (include/gwn/gwn_bvh.cuh:208-258). `node_capacity` is the allocated node count (>= node_count). */
typedef struct gwnb_bvh4_f32 {
    gwnb_node4_f32 *nodes;
    uint64_t node_count;
    uint64_t node_capacity;
    uint32_t *primitive_indices;
    gwnb_triangle_f32 *triangles;
    uint64_t primitive_count;
    gwnb_child_f32 root;
    uint32_t internal_stack_bound;
    uint32_t packed_stack_bound;
    uint64_t revision;
    gwnb_bvh_aux *aux;
} gwnb_bvh4_f32;

typedef struct gwnb_moment_aux gwnb_moment_aux;

/* Device Taylor-moment view; mirrors gwn::gwn_bvh_moment_accessor<4, Order, float, uint32_t>
 * (include/gwn/gwn_bvh.cuh:265-294). `nodes` holds gwn_bvh_moment_node<4, Order, float>. */
typedef struct gwnb_moment4_f32 {
    int order;
    void *nodes;
    uint64_t node_count;
    uint64_t bvh_revision;
    gwnb_moment_aux *aux;
} gwnb_moment4_f32;

/* Options of the Taylor batch beyond smallgwn's template parameters. */
typedef struct gwnb_taylor_options {
    int block_size;     /* smallgwn gwn_query_batch_config::block_size (0 = default 256)        */
    int stack_capacity; /* smallgwn gwn_query_batch_config::stack_capacity (0 = default 64)     */
    int sort_queries;   /* 1: Hilbert-order the batch internally for traversal coherence         */
    int near_precision; /* GWNB_NEAR_PLAIN or GWNB_NEAR_COMPENSATED                               */
    float fp64_threshold; /* compensated mode: |den| < threshold * |a||b||c| takes the FP64 path */
    int per_thread;       /* GWNB_WALK_WARP (0, default), GWNB_WALK_THREAD (1) or GWNB_WALK_TIMED (2) */
} gwnb_taylor_options;

/* ---- status ------------------------------------------------------------------------------ */

/* Message of the most recent failing call on this host thread (smallgwn gwn_status::message,
 * include/gwn/gwn_utils.cuh:212-283). */
GWNB_API const char *gwnb_last_error_message(void);
/* CUDA error code of the most recent GWNB_CUDA_RUNTIME_ERROR on this host thread. */
GWNB_API int gwnb_last_cuda_error(void);
/* Library version string. */
GWNB_API const char *gwnb_version(void);
/* Version of the CUDA runtime the library runs on (1000 * major + 10 * minor; 0 if unknown). */
GWNB_API int gwnb_cuda_runtime_version(void);

/* Number of kernel launches this library has issued in the process (all threads and devices); a
 * launch recorded into a CUDA graph counts once, when it is captured. For benchmarks and tests that
 * check which work ran on the GPU. */
GWNB_API uint64_t gwnb_launch_count(void);

/* Measured FP32 fused-multiply-add throughput of the current device (no smallgwn counterpart): one
 * launch of independent FMA chains on every SM, timed with CUDA events on `stream` after one
 * untimed launch; *tflops = 2 x FMAs / device time, *ms (may be NULL) = that time. The compute
 * roofline of the Taylor traversal, which is bound by instruction issue on the CUDA cores, is
 * reported against it. */
GWNB_API int gwnb_fp32_fma_peak(int iters, double *tflops, double *ms, gwnb_stream_t stream);

/* ---- bounded device waits (no smallgwn counterpart) ----------------------------------------------
 * smallgwn's BVH4 collapse spins without a limit on its work queue (detail/gwn_bvh_build_collapse.cuh
 * :142-144). Every device-side wait of this library -- the decoupled look-back of the radix sort and
 * of the level-synchronous collapse -- gives up after a number of polls, sets a timeout bit in the
 * call's device status word and lets the launch complete; the synchronizing call that reads the
 * status then returns GWNB_INTERNAL_ERROR. */

/* Polls after which a device wait gives up, for launches issued after the call by any thread of
 * the process; polls <= 0 restores the default (2^22, about 10 ms of polling). A small limit lets a
 * test make a wait run out quickly. */
GWNB_API int gwnb_set_wait_limit(int64_t polls);

/* Runs one look-back whose predecessor tile is never published and reports how the wait ended:
 * stage 0 is a real radix-sort pass over two tiles whose first tile is never processed, stage 1
 * the BVH4 collapse's tile-prefix wait on an unpublished tile. Returns GWNB_INTERNAL_ERROR with a
 * "timed out" message once the wait gives up (the expected outcome), after at most the wait limit
 * in polls; synchronizes `stream`. */
GWNB_API int gwnb_wait_timeout_probe(int stage, gwnb_stream_t stream);

/* ---- device memory ------------------------------------------------------------------------- */
/* Every device allocation of the library comes from one memory pool per device that keeps freed
 * memory mapped between host synchronizations (no smallgwn counterpart: smallgwn allocates with
 * the CUDA defaults, which return freed memory to the driver at each synchronization). These two
 * calls act on the current device's pool. */

/* Bytes the pool holds from the driver (*reserved) and bytes in live allocations (*used); either
 * pointer may be NULL. */
GWNB_API int gwnb_memory_stats(uint64_t *reserved, uint64_t *used);

/* Returns cached memory to the driver until the pool holds at most max(keep_bytes, bytes in use).
 * Call it after the stream work that freed the memory has completed. */
GWNB_API int gwnb_memory_trim(uint64_t keep_bytes);

/* Failure injection on the host, for tests of the error paths: after `count` more device
 * allocations of the library succeed, the next one fails as an out-of-memory allocation would
 * (the call returns GWNB_CUDA_RUNTIME_ERROR, cudaErrorMemoryAllocation, "injected failure" in the
 * message); the injection then disarms itself. A negative count disarms it. Process-wide (every
 * thread's allocations count). Returns the count that was armed before this call: -1 when none
 * was, or the injection has fired since. */
GWNB_API int64_t gwnb_fail_allocation_after(int64_t count);

/* ---- geometry (include/gwn/gwn_geometry.cuh:66-90) ---------------------------------------- */

/* Replaces gwn::gwn_upload_geometry (include/gwn/gwn_geometry.cuh:66-72,
 * detail/gwn_geometry_impl.cuh:183-206). Allocates a new view in *out; the caller releases any
 * previous view (staging-and-swap keeps the previous object intact on failure). Synchronizes
 * `stream` to validate indices, as smallgwn does. */
GWNB_API int gwnb_geometry_upload_f32(gwnb_geometry_f32 *out, const float *x, const float *y, const float *z,
                             uint64_t vertex_count, const uint32_t *i0, const uint32_t *i1,
                             const uint32_t *i2, uint64_t triangle_count, gwnb_stream_t stream);

/* Replaces gwn::gwn_update_geometry (include/gwn/gwn_geometry.cuh:85-90). Host positions,
 * asynchronous. */
GWNB_API int gwnb_geometry_update_f32(gwnb_geometry_f32 *geometry, const float *x, const float *y,
                             const float *z, uint64_t vertex_count, gwnb_stream_t stream);

/* Same as gwnb_geometry_update_f32 but the positions already live in device memory. */
GWNB_API int gwnb_geometry_update_device_f32(gwnb_geometry_f32 *geometry, const float *x, const float *y,
                                    const float *z, uint64_t vertex_count, gwnb_stream_t stream);

/* Replaces gwn::detail::gwn_release_accessor (detail/gwn_geometry_impl.cuh:16-26). */
GWNB_API void gwnb_geometry_release_f32(gwnb_geometry_f32 *geometry, gwnb_stream_t stream);

/* ---- BVH build (include/gwn/gwn_bvh_build.cuh:15-39) ------------------------------------- */

/* Replaces gwn::gwn_build_bvh<4, float, uint32_t, MortonCode> (include/gwn/gwn_bvh_build.cuh:34-39,
 * detail/gwn_bvh_build_impl.cuh:44-274). method: GWNB_METHOD_HPLOC or GWNB_METHOD_LBVH;
 * hploc_search_radius in [1, 8]; morton_bits 32 or 64. Writes a new view into *out. */
GWNB_API int gwnb_bvh4_build_f32(const gwnb_geometry_f32 *geometry, int method, uint32_t hploc_search_radius,
                        int morton_bits, gwnb_bvh4_f32 *out, gwnb_stream_t stream);

/* Replaces gwn::detail::gwn_release_bvh_accessor (include/gwn/gwn_bvh.cuh:301-313). */
GWNB_API void gwnb_bvh4_release_f32(gwnb_bvh4_f32 *bvh, gwnb_stream_t stream);

/* Build stages exposed for parity checks. Output buffers are caller-owned device memory sized
 * for triangle_count elements (binary arrays: triangle_count - 1).
 * Replaces gwn::detail::gwn_bvh_build_preprocess (detail/gwn_bvh_build_common.cuh:371-381):
 * sorted Morton codes (uint32 or uint64 per morton_bits), sorted primitive ids, sorted AABBs. */
GWNB_API int gwnb_build_preprocess_f32(const gwnb_geometry_f32 *geometry, int morton_bits,
                              void *sorted_codes, uint32_t *sorted_ids, gwnb_aabb_f32 *sorted_aabbs,
                              gwnb_stream_t stream);

/* Binary node as produced by the binary builders: (left index, left kind, right index, right
 * kind), kind 1 = internal, 2 = leaf (detail/gwn_bvh_build_binary.cuh:13-28). */
typedef struct gwnb_binary_node {
    uint32_t left_index;
    uint32_t left_kind;
    uint32_t right_index;
    uint32_t right_kind;
} gwnb_binary_node;

/* Replaces gwn::detail::gwn_bvh_build_binary_lbvh (detail/gwn_bvh_build_lbvh.cuh:19-99). */
GWNB_API int gwnb_build_binary_lbvh(const void *sorted_codes, int morton_bits, uint64_t count,
                           const gwnb_aabb_f32 *sorted_aabbs, gwnb_binary_node *nodes,
                           uint32_t *internal_parent, gwnb_aabb_f32 *internal_bounds,
                           gwnb_stream_t stream);

/* Replaces gwn::detail::gwn_bvh_build_binary_hploc_impl (detail/gwn_bvh_build_hploc.cuh:480-622).
 * Writes the root internal index to *root (device-to-host copy, synchronizes). */
GWNB_API int gwnb_build_binary_hploc(const void *sorted_codes, int morton_bits, uint64_t count,
                            const gwnb_aabb_f32 *sorted_aabbs, uint32_t search_radius,
                            gwnb_binary_node *nodes, uint32_t *internal_parent,
                            gwnb_aabb_f32 *internal_bounds, uint32_t *root, gwnb_stream_t stream);

/* Stable LSD radix sort of (key, value) pairs over key bits [0, key_bits); onesweep passes.
 * Stands in for cub::DeviceRadixSort::SortPairs at detail/gwn_bvh_build_common.cuh:332-347.
 * keys are uint32 (key_bytes 4) or uint64 (key_bytes 8). values may be NULL (identity ids).
 * Results go to keys_out / values_out. */
GWNB_API int gwnb_radix_sort_pairs(const void *keys_in, void *keys_out, const uint32_t *values_in,
                          uint32_t *values_out, uint64_t count, int key_bytes, int key_bits,
                          gwnb_stream_t stream);

/* ---- refit (include/gwn/gwn_bvh_refit.cuh:25-51) ----------------------------------------- */

/* Replaces gwn::gwn_refit_bvh (include/gwn/gwn_bvh_refit.cuh:25-29,
 * detail/gwn_bvh_refit_impl.cuh:194-352). Synchronizes to publish root bounds and errors, as
 * smallgwn does. */
GWNB_API int gwnb_bvh4_refit_f32(const gwnb_geometry_f32 *geometry, gwnb_bvh4_f32 *bvh, gwnb_stream_t stream);

/* Stream-ordered refit with no host synchronization and no allocation after the first call on a
 * BVH (capturable in a CUDA graph). Root bounds and errors stay on the device; read them with
 * gwnb_bvh4_sync_status_f32. Has no smallgwn counterpart (smallgwn's refit always synchronizes). */
GWNB_API int gwnb_bvh4_refit_async_f32(const gwnb_geometry_f32 *geometry, gwnb_bvh4_f32 *bvh,
                              gwnb_stream_t stream);

/* Synchronizes `stream`, copies the device-side root bounds into bvh->root.bounds and turns the
 * device error word into a status. */
GWNB_API int gwnb_bvh4_sync_status_f32(gwnb_bvh4_f32 *bvh, gwnb_stream_t stream);

/* Replaces gwn::gwn_refit_bvh_moment<Order> (include/gwn/gwn_bvh_refit.cuh:36-51,
 * detail/gwn_bvh_refit_moment_impl.cuh:137-279). Writes a new view into *out. */
GWNB_API int gwnb_moment4_refit_f32(const gwnb_bvh4_f32 *bvh, int order, gwnb_moment4_f32 *out,
                           gwnb_stream_t stream);

/* Refit moments into an existing moment view (same BVH topology, new geometry) without
 * allocation or host synchronization. Has no smallgwn counterpart. */
GWNB_API int gwnb_moment4_refit_async_f32(const gwnb_bvh4_f32 *bvh, gwnb_moment4_f32 *moment,
                                 gwnb_stream_t stream);

/* Replaces gwn::detail::gwn_release_bvh_moment_accessor (include/gwn/gwn_bvh.cuh:316-322). */
GWNB_API void gwnb_moment4_release_f32(gwnb_moment4_f32 *moment, gwnb_stream_t stream);

/* Size in bytes of one gwn_bvh_moment_node<4, order, float>. */
GWNB_API uint64_t gwnb_moment_node_bytes(int order);

/* ---- queries (include/gwn/gwn_query.cuh) -------------------------------------------------- */

/* Replaces gwn::gwn_compute_winding_number_exact_batch<Config> (include/gwn/gwn_query.cuh:308-346).
 * query_* and output are device pointers of `count` floats. Asynchronous. */
GWNB_API int gwnb_winding_exact_batch_f32(const gwnb_bvh4_f32 *bvh, const float *query_x,
                                 const float *query_y, const float *query_z, float *output,
                                 uint64_t count, int block_size, gwnb_stream_t stream);

/* Replaces gwn::gwn_compute_winding_number_taylor_batch<Order, Config>
 * (include/gwn/gwn_query.cuh:384-445). `options` may be NULL (defaults: block 256, stack 64,
 * sorted queries, plain near field). Asynchronous. A traversal that would overflow its stack
 * writes NaN and sets the BVH's device error word instead of trapping. */
GWNB_API int gwnb_winding_taylor_batch_f32(const gwnb_bvh4_f32 *bvh, const gwnb_moment4_f32 *moment,
                                  const float *query_x, const float *query_y, const float *query_z,
                                  float *output, uint64_t count, float accuracy_scale,
                                  const gwnb_taylor_options *options, gwnb_stream_t stream);

/* Replaces gwn::gwn_compute_winding_gradient_taylor_batch<Order, Config>
 * (include/gwn/gwn_query.cuh:688-756): dw/dq of the Taylor winding number. */
GWNB_API int gwnb_winding_gradient_taylor_batch_f32(const gwnb_bvh4_f32 *bvh,
                                           const gwnb_moment4_f32 *moment, const float *query_x,
                                           const float *query_y, const float *query_z,
                                           float *grad_x, float *grad_y, float *grad_z,
                                           uint64_t count, float accuracy_scale,
                                           const gwnb_taylor_options *options,
                                           gwnb_stream_t stream);

/* Per-query traversal statistics of the Taylor batch (diagnostics; nodes entered, far-field
 * child evaluations, exact near-field triangles). Writes three uint32 arrays of `count`. */
GWNB_API int gwnb_winding_taylor_stats_f32(const gwnb_bvh4_f32 *bvh, const gwnb_moment4_f32 *moment,
                                  const float *query_x, const float *query_y, const float *query_z,
                                  uint64_t count, float accuracy_scale, uint32_t *nodes_entered,
                                  uint32_t *far_evaluations, uint32_t *near_triangles,
                                  gwnb_stream_t stream);

/* Sampled walk statistics of a Taylor batch (diagnostics; which of the two traversals suits it):
 * orders the batch as the Taylor batch would (options' sort_queries), walks a sample of it
 * warp-cooperatively with statistics and no outputs (every k-th unit of 32 consecutive ordered
 * warps: one resident wave or 1/64 of the batch, up to 64 units for small batches) and writes, per
 * sampled warp, out[0] nodes the warp walked, out[1]
 * leaf triangles it evaluated, out[2] the largest per-query node count and out[3] the largest
 * per-query triangle count in the warp; out[4] the sampled warps (0 below 1,024 queries); out[5] 1
 * when the per-thread traversal suits the batch (sampled warps walked at least 1.3 times their
 * longest path's nodes, that path met at most 8 leaf triangles). Synchronizes `stream`. */
GWNB_API int gwnb_taylor_form_probe_f32(const gwnb_bvh4_f32 *bvh, const gwnb_moment4_f32 *moment,
                                        const float *query_x, const float *query_y, const float *query_z,
                                        uint64_t count, float accuracy_scale, const gwnb_taylor_options *options,
                                        double *out, gwnb_stream_t stream);

/* ---- Taylor order and accuracy scale from an error target (no smallgwn counterpart) ------------
 * smallgwn leaves the Taylor order (a template parameter) and the accuracy scale to the caller. */

typedef struct gwnb_taylor_choice {
    int order;              /* chosen Taylor order                                               */
    float accuracy_scale;   /* chosen beta                                                       */
    float max_error;        /* max |w - w_fp64| over the sample with that choice                 */
    float sample_ms;        /* device time of one Taylor batch over the sample with that choice  */
    int stack_capacity;     /* traversal stack the tree needs: its exact internal stack bound    */
    int candidates_passing; /* orders with some candidate beta within the bound                  */
} gwnb_taylor_choice;

/* Picks the Taylor order and accuracy scale for a caller's error bound on a sample of the caller's
 * queries (device arrays qx/qy/qz of n): the sample's FP64 exact winding numbers are the reference;
 * for every order o whose moments[o] is non-NULL (valid for `bvh`), the smallest of the candidate
 * `betas` whose maximum error on the sample is at most max_error is that order's candidate; the
 * candidates are timed on the sample (CUDA events, same stream) and the fastest is returned in *out.
 * GWNB_INVALID_ARGUMENT when no candidate meets the bound. Synchronizes `stream`. */
GWNB_API int gwnb_taylor_select_f32(const gwnb_geometry_f32 *geometry, const gwnb_bvh4_f32 *bvh,
                                    const gwnb_moment4_f32 *const *moments, const float *qx, const float *qy,
                                    const float *qz, uint64_t n, float max_error, const float *betas,
                                    int beta_count, int near_precision, gwnb_taylor_choice *out,
                                    gwnb_stream_t stream);

/* Exact winding numbers of the float mesh evaluated in FP64 (brute force over the geometry's
 * triangles, double-precision Van Oosterom-Strackee). Counterpart of smallgwn's Real = double
 * instantiation of gwn_compute_winding_number_exact_batch (tests/reference_cpu.cuh:84-114 is its
 * CPU form); used as the FP64 error reference. query_* are float, output is double. */
GWNB_API int gwnb_winding_exact_geometry_fp64(const gwnb_geometry_f32 *geometry, const float *query_x,
                                              const float *query_y, const float *query_z, double *output,
                                              uint64_t count, gwnb_stream_t stream);

/* ---- spatial queries (include/gwn/gwn_query.cuh:63-282) ----------------------------------- */

/* Launch options of the distance and ray batches (smallgwn gwn_query_batch_config plus ordering). */
typedef struct gwnb_spatial_options {
    int block_size;     /* gwn_query_batch_config::block_size, multiple of 32 (0 = default 256)  */
    int stack_capacity; /* gwn_query_batch_config::stack_capacity (0 = default 64)               */
    int sort_queries;   /* 1: traverse in Hilbert order of the query points / ray origins        */
    int per_thread;     /* distance batches in Hilbert order: GWNB_WALK_WARP (0, default),
                         * GWNB_WALK_THREAD (1) or GWNB_WALK_TIMED (2); identical results           */
} gwnb_spatial_options;
/* Distance batches in Hilbert order are walked warp-cooperatively (32 neighbouring queries walk one
 * traversal, each lane pruning by its own bound) or one query per thread; in input order, and every
 * ray batch, run persistently: a thread whose query has finished takes the next unclaimed one. For
 * the rays of the 1M-triangle benchmark, input order (sort_queries = 0) is the faster choice. */

/* gwn::gwn_ray_first_hit_status (include/gwn/gwn_query.cuh:63-68). */
enum { GWNB_RAY_MISS = 0, GWNB_RAY_HIT = 1, GWNB_RAY_OVERFLOW = 2 };

/* Layout of gwn::gwn_ray_first_hit_result<float, uint32_t> (include/gwn/gwn_query.cuh:70-96),
 * 32 bytes. A miss has t = -1, primitive_id = 0xffffffff and zero weights and normal. */
typedef struct gwnb_ray_hit_f32 {
    float t;                  /* ray parameter of the hit                                   */
    float u, v;               /* barycentric weights of the second and third vertex          */
    float geometric_normal_x; /* unnormalized oriented geometric normal                      */
    float geometric_normal_y;
    float geometric_normal_z;
    uint32_t primitive_id; /* original mesh primitive id                                   */
    uint8_t status;        /* GWNB_RAY_MISS, GWNB_RAY_HIT or GWNB_RAY_OVERFLOW             */
    uint8_t padding[3];    /* zero                                                          */
} gwnb_ray_hit_f32;

/* Replaces gwn::gwn_compute_unsigned_distance_batch<Config> (include/gwn/gwn_query.cuh:135-183,
 * detail/gwn_query_distance_impl.cuh:40-160): distance of each query point to the nearest
 * triangle, at most `culling_band` (negative bands clamp to 0, infinity searches unbounded).
 * `options` may be NULL (block 256, stack 64, input order). Asynchronous. A traversal that would
 * overflow its stack writes NaN and sets the BVH's device error word instead of trapping. */
GWNB_API int gwnb_unsigned_distance_batch_f32(const gwnb_bvh4_f32 *bvh, const float *query_x,
                                              const float *query_y, const float *query_z, float *output,
                                              uint64_t count, float culling_band,
                                              const gwnb_spatial_options *options, gwnb_stream_t stream);

/* Replaces gwn::gwn_compute_ray_first_hit_batch<Config> (include/gwn/gwn_query.cuh:214-282,
 * detail/gwn_query_ray_impl.cuh:376-560): nearest hit of each ray on the closed interval
 * [t_min, t_max] (t_max >= t_min required). Among hits at the same t the lower primitive id is
 * reported. Asynchronous. */
GWNB_API int gwnb_ray_first_hit_batch_f32(const gwnb_bvh4_f32 *bvh, const float *ray_origin_x,
                                          const float *ray_origin_y, const float *ray_origin_z,
                                          const float *ray_dir_x, const float *ray_dir_y, const float *ray_dir_z,
                                          gwnb_ray_hit_f32 *output, uint64_t count, float t_min, float t_max,
                                          const gwnb_spatial_options *options, gwnb_stream_t stream);

enum { GWNB_SPATIAL_DISTANCE = 0, GWNB_SPATIAL_RAY = 1 };

/* Per-query traversal statistics of a distance (kind GWNB_SPATIAL_DISTANCE; dir_* unused) or ray
 * batch (GWNB_SPATIAL_RAY): internal nodes entered and triangles tested, two uint32 arrays of
 * `count` (diagnostics behind the benchmark's bytes model). No smallgwn counterpart. */
GWNB_API int gwnb_spatial_stats_f32(const gwnb_bvh4_f32 *bvh, int kind, const float *query_x, const float *query_y,
                                    const float *query_z, const float *dir_x, const float *dir_y,
                                    const float *dir_z, uint64_t count, float culling_band, float t_min,
                                    float t_max, uint32_t *nodes_entered, uint32_t *triangles_tested,
                                    gwnb_stream_t stream);

/* ---- boundary chain and antipodal winding numbers (include/gwn/gwn_boundary.cuh,
 *      include/gwn/gwn_query.cuh:446-656) ------------------------------------------------------ */

/* Device boundary chain; mirrors gwn::gwn_boundary_chain_accessor<uint32_t>
 * (include/gwn/gwn_boundary.cuh:22-59): directed boundary edges (start, end vertex) with their
 * positive net multiplicity, rows in ascending (low vertex, high vertex) order. */
typedef struct gwnb_boundary_chain_u32 {
    uint32_t *start_vertex;
    uint32_t *end_vertex;
    uint64_t *multiplicity;
    uint64_t edge_count;
    uint64_t mesh_vertex_count;   /* vertex count of the mesh the chain was built from   */
    uint64_t mesh_triangle_count; /* triangle count of the mesh the chain was built from */
    int is_built;                 /* 1 after a successful build, closed meshes included   */
} gwnb_boundary_chain_u32;

/* Replaces gwn::gwn_build_boundary_chain (include/gwn/gwn_boundary.cuh:116-125,
 * detail/gwn_boundary_impl.cuh:182-415): the algebraic boundary of the oriented triangle chain.
 * Writes a new chain into *out (the caller releases any previous one). Synchronizes `stream` once
 * to size the output, as smallgwn does. */
GWNB_API int gwnb_boundary_chain_build_u32(const gwnb_geometry_f32 *geometry, gwnb_boundary_chain_u32 *out,
                                           gwnb_stream_t stream);

/* Replaces gwn::detail::gwn_release_boundary_chain_accessor (detail/gwn_boundary_impl.cuh:98-110). */
GWNB_API void gwnb_boundary_chain_release_u32(gwnb_boundary_chain_u32 *chain, gwnb_stream_t stream);

/* Replaces gwn::gwn_compute_winding_number_antipodal_batch<Config> (include/gwn/gwn_query.cuh:
 * 497-556): signed crossings of the +z (then +x, +y) coordinate ray through the BVH plus the
 * boundary spherical-area term; NaN where all three axes are singular. `options` may be NULL
 * (block 256, stack 64, input order; sort_queries = 1 traverses in Hilbert order). Asynchronous. */
GWNB_API int gwnb_winding_antipodal_batch_f32(const gwnb_geometry_f32 *geometry, const gwnb_bvh4_f32 *bvh,
                                              const gwnb_boundary_chain_u32 *chain, const float *query_x,
                                              const float *query_y, const float *query_z, float *output,
                                              uint64_t count, const gwnb_spatial_options *options,
                                              gwnb_stream_t stream);

/* Replaces gwn::gwn_compute_winding_gradient_antipodal_batch<Config> (include/gwn/gwn_query.cuh:
 * 596-654): gradient of the boundary term; (NaN, NaN, NaN) where all three axes are singular.
 * block_size 0 selects 256. Asynchronous. */
GWNB_API int gwnb_winding_gradient_antipodal_batch_f32(const gwnb_geometry_f32 *geometry,
                                                       const gwnb_boundary_chain_u32 *chain, const float *query_x,
                                                       const float *query_y, const float *query_z, float *grad_x,
                                                       float *grad_y, float *grad_z, uint64_t count, int block_size,
                                                       gwnb_stream_t stream);

/* Traversal order of a ray batch (the permutation the ray batch applies when sort_queries is
 * set): rays sorted by the octahedral cell of their direction, then by the Hilbert index of their
 * origin relative to the BVH root bounds. order[i] is the index of the i-th ray. No smallgwn
 * counterpart. */
GWNB_API int gwnb_ray_order_f32(const gwnb_bvh4_f32 *bvh, const float *ray_origin_x, const float *ray_origin_y,
                                const float *ray_origin_z, const float *ray_dir_x, const float *ray_dir_y,
                                const float *ray_dir_z, uint64_t count, uint32_t *order, gwnb_stream_t stream);

/* Hilbert order of a query batch relative to the BVH root bounds: order[i] is the index of the
 * i-th query in traversal-coherent order (the permutation the Taylor batch applies internally when
 * sort_queries is set). No smallgwn counterpart. */
GWNB_API int gwnb_query_order_f32(const gwnb_bvh4_f32 *bvh, const float *query_x, const float *query_y,
                                  const float *query_z, uint64_t count, uint32_t *order, gwnb_stream_t stream);

/* ---- mesh and scene files ------------------------------------------------------------------ */

/* Host triangle mesh (SoA): what smallgwn's tests load into their HostMesh
 * (tests/test_mesh_io.hpp). Arrays from gwnb_mesh_read_ply are malloc'd; free them with
 * gwnb_host_mesh_free. */
typedef struct gwnb_host_mesh_f32 {
    float *x, *y, *z;
    uint64_t vertex_count;
    uint32_t *i0, *i1, *i2;
    uint64_t triangle_count;
} gwnb_host_mesh_f32;

/* Replaces smallgwn's test helper gwn::tests::load_ply_mesh (tests/test_mesh_io.cpp:43-92, libigl's
 * reader): ASCII or binary (either byte order) PLY with any numeric property types; vertex x, y, z
 * narrowed to float; the face index list ("vertex_indices", else the face element's first list)
 * with polygons split into triangle fans. Refuses non-finite positions, out-of-range indices,
 * faces with fewer than three vertices and meshes without vertices or triangles. */
GWNB_API int gwnb_mesh_read_ply(const char *path, gwnb_host_mesh_f32 *out);

/* Frees the arrays of a mesh read by gwnb_mesh_read_ply and zeroes it. */
GWNB_API void gwnb_host_mesh_free(gwnb_host_mesh_f32 *mesh);

/* Writes a host mesh as PLY (float positions, uint32 index lists); binary = 1 for
 * binary_little_endian, 0 for ASCII. No smallgwn counterpart. */
GWNB_API int gwnb_mesh_write_ply(const char *path, const gwnb_host_mesh_f32 *mesh, int binary);

/* Saves geometry, BVH and up to three moment objects (one per order) in one file, so that a later
 * process skips the build (no smallgwn counterpart: smallgwn rebuilds every run). Synchronizes
 * `stream`. */
GWNB_API int gwnb_scene_save_f32(const char *path, const gwnb_geometry_f32 *geometry, const gwnb_bvh4_f32 *bvh,
                                 const gwnb_moment4_f32 *const *moments, int moment_count, gwnb_stream_t stream);

/* Loads a scene file: new geometry and BVH views (a fresh revision) and, for every moment order
 * saved in the file, a moment view in moments[order] refit from the loaded BVH and checked equal to
 * the saved nodes. *moment_mask (may be NULL) receives the saved orders as bits 0-2. Refuses
 * files with a bad magic, version or checksum. Synchronizes `stream`. */
GWNB_API int gwnb_scene_load_f32(const char *path, gwnb_geometry_f32 *geometry, gwnb_bvh4_f32 *bvh,
                                 gwnb_moment4_f32 moments[3], int *moment_mask, gwnb_stream_t stream);

/* Largest batch gwnb_winding_taylor_batch_noalloc_f32 accepts. */
#define GWNB_NOALLOC_MAX_QUERIES 262144u

/* Taylor batch that allocates no device memory (no smallgwn counterpart: smallgwn's batches need
 * no scratch, this library's allocate their query-ordering scratch per call). For callers that
 * cannot let a library allocate -- fixed device-memory budgets owned by a host engine, real-time
 * loops where an allocation would stall, replayed work that forbids new allocations. Same
 * arguments and results as gwnb_winding_taylor_batch_f32; at most GWNB_NOALLOC_MAX_QUERIES
 * queries per call (larger batches return GWNB_INVALID_ARGUMENT). Scratch is one file-scope
 * device array (about 5.5 MB) that every GPU loading the library holds until exit; calls whose
 * work overlaps on the GPU race on it. The BVH must already carry derived state (built or refit
 * by this library). The first call on a device looks up the array's address; make it before any
 * stream capture. options->per_thread takes GWNB_WALK_WARP or GWNB_WALK_THREAD only (the timed
 * choice keeps events, which a call that allocates nothing does not create). */
GWNB_API int gwnb_winding_taylor_batch_noalloc_f32(const gwnb_bvh4_f32 *bvh, const gwnb_moment4_f32 *moment,
                                                   const float *query_x, const float *query_y,
                                                   const float *query_z, float *output, uint64_t count,
                                                   float accuracy_scale, const gwnb_taylor_options *options,
                                                   gwnb_stream_t stream);

/* Number of FP64 fallbacks taken by the last compensated Taylor batch on this BVH (device
 * counter read back with a synchronization). */
GWNB_API int gwnb_bvh4_fp64_fallback_count(const gwnb_bvh4_f32 *bvh, uint64_t *count, gwnb_stream_t stream);

/* ---- adjoint of the Taylor batch (no smallgwn counterpart) --------------------------------- */

/* What a forward pass keeps for its backward pass -- the save-for-backward contract a
 * torch.autograd.Function wraps: the query arrays by reference (the caller keeps them alive and
 * unchanged until the backward call) and the BVH revision the result was computed at. No
 * traversal state is kept; the backward pass recomputes the traversal. */
typedef struct gwnb_taylor_saved_f32 {
    const float *query_x;
    const float *query_y;
    const float *query_z;
    uint64_t count;
    float accuracy_scale;
    int order;
    uint64_t bvh_revision;
    gwnb_taylor_options options;
} gwnb_taylor_saved_f32;

/* Forward: the Taylor batch of gwnb_winding_taylor_batch_f32 (orders 0 and 1 only), filling
 * `saved` for gwnb_winding_taylor_backward_f32. */
GWNB_API int gwnb_winding_taylor_forward_f32(const gwnb_bvh4_f32 *bvh, const gwnb_moment4_f32 *moment,
                                             const float *query_x, const float *query_y, const float *query_z,
                                             float *output, uint64_t count, float accuracy_scale,
                                             const gwnb_taylor_options *options, gwnb_taylor_saved_f32 *saved,
                                             gwnb_stream_t stream);

/* Backward: given grad_output g (count floats), the gradients of L = sum_q g_q w(q) with respect to
 * the geometry's vertex positions (grad_vertex_*: vertex_count floats each, overwritten) and the
 * query points (grad_query_*: count floats each). Either triple may be all NULL to skip it. The
 * BVH must be the one of the forward pass at the same revision, built from `geometry` (one
 * primitive per geometry triangle), with `moment` refit for it. Acceptance decisions are held
 * fixed (they carry no derivative); slots of zero area pass no gradient through their centre.
 * Asynchronous on `stream`. */
GWNB_API int gwnb_winding_taylor_backward_f32(const gwnb_taylor_saved_f32 *saved, const gwnb_geometry_f32 *geometry,
                                              const gwnb_bvh4_f32 *bvh, const gwnb_moment4_f32 *moment,
                                              const float *grad_output, float *grad_vertex_x,
                                              float *grad_vertex_y, float *grad_vertex_z, float *grad_query_x,
                                              float *grad_query_y, float *grad_query_z, gwnb_stream_t stream);

/* ---- batched dynamic meshes (no smallgwn counterpart) ----------------------------------------- */

/* Many meshes whose vertices move every frame (topology fixed): one frame refits every BVH and its
 * moments and evaluates every mesh's Taylor queries in three persistent launches, with no host
 * synchronization, so a frame can be captured in a CUDA graph. */
typedef struct gwnb_batch gwnb_batch;

typedef struct gwnb_batch_mesh_f32 {
    gwnb_geometry_f32 geometry; /* view of the mesh (positions read by every frame's refit)      */
    gwnb_bvh4_f32 *bvh;         /* built by this library from `geometry`; refit in place          */
    gwnb_moment4_f32 *moment;   /* moments of `bvh`; refit in place (all meshes share one order)  */
    const float *query_x;       /* this mesh's queries (fixed for the batch; read every frame)    */
    const float *query_y;
    const float *query_z;
    float *output;              /* winding numbers, query_count floats                            */
    uint64_t query_count;
} gwnb_batch_mesh_f32;

/* Launch shape of a frame, as chosen by gwnb_batch_tune_f32. */
typedef struct gwnb_batch_tuning {
    int refit_block;  /* threads per block of the refit launches                                  */
    int query_block;  /* threads per block of the query launch (multiple of 32, at most 256)      */
    int per_thread;   /* 0: 32 queries per warp walk one traversal; 1: one traversal per thread   */
    int sorted;       /* 1: traverse each mesh's queries in Hilbert order (computed at creation)  */
    int grid_scale;   /* persistent grids of SMs x grid_scale blocks                              */
    float frame_ms;   /* measured frame time of this shape (output of tuning)                     */
} gwnb_batch_tuning;

/* Creates a batch over `mesh_count` meshes (copies the descriptors; the pointed-to objects must
 * outlive the batch). Computes each mesh's query order. While the batch exists its frames refit the
 * BVHs and moments in place and leave their revisions unchanged. A BVH or moment object given new
 * arrays outside the batch (built again, moments refit into it) makes every later call on the
 * batch except release return GWNB_INVALID_ARGUMENT. */
GWNB_API int gwnb_batch_create_f32(const gwnb_batch_mesh_f32 *meshes, uint32_t mesh_count, float accuracy_scale,
                                   const gwnb_taylor_options *options, gwnb_batch **batch, gwnb_stream_t stream);
/* Times `repetitions` frames of every candidate launch shape on `stream` and keeps the fastest
 * (written to `chosen` when non-NULL). Frames run: the meshes are refit and queried. */
GWNB_API int gwnb_batch_tune_f32(gwnb_batch *batch, int repetitions, gwnb_batch_tuning *chosen, gwnb_stream_t stream);
GWNB_API int gwnb_batch_set_tuning_f32(gwnb_batch *batch, const gwnb_batch_tuning *tuning);
/* Enqueues one frame (refit, moment refit, queries) on `stream`; asynchronous and capturable once
 * a frame or a tuning has run outside capture. */
GWNB_API int gwnb_batch_frame_f32(gwnb_batch *batch, gwnb_stream_t stream);

/* Stages of a frame, for gwnb_batch_run_f32 (a frame is all three, in this order). */
#define GWNB_BATCH_REFIT 1u   /* bounds and triangle records of every BVH                */
#define GWNB_BATCH_MOMENTS 2u /* Taylor moments of every BVH (after the bounds)          */
#define GWNB_BATCH_QUERY 4u   /* every mesh's Taylor queries                             */
/* Enqueues the selected stages of a frame (e.g. refit once, then query several times). */
GWNB_API int gwnb_batch_run_f32(gwnb_batch *batch, unsigned int stages, gwnb_stream_t stream);
/* Synchronizes `stream` and reports device-side errors of any mesh (index or topology faults,
 * stack overflow) as GWNB_INTERNAL_ERROR. */
GWNB_API int gwnb_batch_sync_f32(gwnb_batch *batch, gwnb_stream_t stream);
GWNB_API int gwnb_batch_release_f32(gwnb_batch *batch, gwnb_stream_t stream);

/* Tree quality (no smallgwn counterpart): per mesh, the surface-area cost of its BVH now -- the sum
 * over nodes of the children's box half-areas over the root box's half-area -- divided by that cost
 * when the tree was built (cost_ratio: mesh_count floats, host). Refitting keeps the rest shape's
 * topology, so the ratio grows as the meshes deform and queries visit more nodes. Synchronizes. */
GWNB_API int gwnb_batch_quality_f32(gwnb_batch *batch, float *cost_ratio, gwnb_stream_t stream);

/* Rebuilds (method, radius as gwnb_bvh4_build_f32, 64-bit Morton codes) every BVH whose cost ratio
 * exceeds `threshold`, from its geometry's current positions, refits its moments, replaces the
 * caller's BVH and moment objects in place and re-derives the batch's descriptors (*rebuilt: how
 * many). Between frames: a CUDA graph captured before a rebuild that rebuilt anything refers to the
 * released arrays and must be captured again. On failure the meshes rebuilt so far keep their new
 * objects; if the descriptors could not be derived again, frames, stage runs, tuning and sync
 * return GWNB_INTERNAL_ERROR ("incomplete") until a later rebuild call derives them. Synchronizes. */
GWNB_API int gwnb_batch_rebuild_f32(gwnb_batch *batch, float threshold, int method, uint32_t radius,
                                    uint32_t *rebuilt, gwnb_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* GWNB_H */
