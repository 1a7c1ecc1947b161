// ref_shim.cu -- extern "C" shim over smallgwn's own CUDA implementation (TEST INFRASTRUCTURE).
//
// Compiled by oracle/build.py against smallgwn's headers where they lie (never copied into this
// repository) into oracle/_ref/libgwnref.so. Parity tests call it to obtain the reference
// project's own outputs -- Morton codes, sorted permutation, binary topology, wide BVH, moments,
// exact / Taylor winding numbers and the FP64 exact instantiation -- on the same inputs the CUDA
// library receives, and to time its kernels on the same GPU. Nothing in the product path loads it.
//
// Host arrays in, host arrays out; everything runs on the legacy default stream.
#include <gwn/detail/gwn_bvh_build_binary.cuh>
#include <gwn/detail/gwn_bvh_build_common.cuh>
#include <gwn/detail/gwn_bvh_build_hploc.cuh>
#include <gwn/detail/gwn_bvh_build_lbvh.cuh>
#include <gwn/detail/gwn_device_array.cuh>
#include <gwn/gwn.cuh>

#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

namespace {

using Real = float;
using Index = std::uint32_t;

thread_local std::string g_msg;

int fail(gwn::gwn_status const &s) {
    g_msg = s.message();
    return static_cast<int>(s.error());
}

struct no_trap {
    __device__ void operator()() const noexcept {}
};

template <class T> struct dbuf;

struct ctx {
    gwn::gwn_geometry_object<Real, Index> geometry;
    gwn::gwn_bvh4_object<Real, Index> bvh;
    gwn::gwn_bvh4_moment_object<0, Real, Index> m0;
    gwn::gwn_bvh4_moment_object<1, Real, Index> m1;
    gwn::gwn_bvh4_moment_object<2, Real, Index> m2;
    gwn::gwn_boundary_chain_object<Index> chain;
    // device-resident query batch of the dynamic frame (ref_set_queries / ref_dynamic_frame)
    std::unique_ptr<dbuf<float>> qx, qy, qz, out;
};

template <class T> struct dbuf {
    T *p = nullptr;
    std::size_t n = 0;
    explicit dbuf(std::size_t count) : n(count) {
        if (count)
            cudaMalloc(&p, count * sizeof(T));
    }
    dbuf(T const *host, std::size_t count) : dbuf(count) {
        if (count)
            cudaMemcpy(p, host, count * sizeof(T), cudaMemcpyHostToDevice);
    }
    ~dbuf() {
        if (p)
            cudaFree(p);
    }
    void to_host(T *host) const {
        if (n)
            cudaMemcpy(host, p, n * sizeof(T), cudaMemcpyDeviceToHost);
    }
};

template <int Order, gwn::gwn_query_batch_config Config>
gwn::gwn_status taylor_cfg(ctx &c, gwn::gwn_bvh4_moment_object<Order, Real, Index> const &m, dbuf<float> &x,
                           dbuf<float> &y, dbuf<float> &z, dbuf<float> &o, float beta) {
    return gwn::gwn_compute_winding_number_taylor_batch<Order, Config, 4, Real, Index, no_trap>(
        c.bvh, m, gwn::gwn_device_span<float const>(x.p, x.n), gwn::gwn_device_span<float const>(y.p, y.n),
        gwn::gwn_device_span<float const>(z.p, z.n), gwn::gwn_device_span<float>(o.p, o.n), beta,
        gwn::gwn_default_stream(), no_trap{});
}

template <int Order>
gwn::gwn_status taylor_any(ctx &c, gwn::gwn_bvh4_moment_object<Order, Real, Index> const &m, dbuf<float> &x,
                           dbuf<float> &y, dbuf<float> &z, dbuf<float> &o, float beta) {
    if (c.bvh.accessor().internal_stack_bound <= 64)
        return taylor_cfg<Order, gwn::gwn_query_batch_config{256, 64}>(c, m, x, y, z, o, beta);
    return taylor_cfg<Order, gwn::gwn_query_batch_config{256, 256}>(c, m, x, y, z, o, beta);
}

template <int Order>
gwn::gwn_status gradient_any(ctx &c, gwn::gwn_bvh4_moment_object<Order, Real, Index> const &m, dbuf<float> &x,
                             dbuf<float> &y, dbuf<float> &z, dbuf<float> &gx, dbuf<float> &gy, dbuf<float> &gz,
                             float beta) {
    constexpr gwn::gwn_query_batch_config cfg{256, 64};
    return gwn::gwn_compute_winding_gradient_taylor_batch<Order, cfg, 4, Real, Index, no_trap>(
        c.bvh, m, gwn::gwn_device_span<float const>(x.p, x.n), gwn::gwn_device_span<float const>(y.p, y.n),
        gwn::gwn_device_span<float const>(z.p, z.n), gwn::gwn_device_span<float>(gx.p, gx.n),
        gwn::gwn_device_span<float>(gy.p, gy.n), gwn::gwn_device_span<float>(gz.p, gz.n), beta,
        gwn::gwn_default_stream(), no_trap{});
}

gwn::gwn_status taylor_order(ctx &c, int order, dbuf<float> &x, dbuf<float> &y, dbuf<float> &z, dbuf<float> &o,
                             float beta) {
    if (order == 0)
        return taylor_any<0>(c, c.m0, x, y, z, o, beta);
    if (order == 1)
        return taylor_any<1>(c, c.m1, x, y, z, o, beta);
    return taylor_any<2>(c, c.m2, x, y, z, o, beta);
}

using ray_result = gwn::gwn_ray_first_hit_result<Real, Index>;
static_assert(sizeof(ray_result) == 32, "smallgwn's ray record is 32 bytes");

template <gwn::gwn_query_batch_config Config>
gwn::gwn_status distance_cfg(ctx &c, dbuf<float> &x, dbuf<float> &y, dbuf<float> &z, dbuf<float> &o, float band) {
    return gwn::gwn_compute_unsigned_distance_batch<Config, 4, Real, Index, no_trap>(
        c.bvh, gwn::gwn_device_span<float const>(x.p, x.n), gwn::gwn_device_span<float const>(y.p, y.n),
        gwn::gwn_device_span<float const>(z.p, z.n), gwn::gwn_device_span<float>(o.p, o.n), band,
        gwn::gwn_default_stream(), no_trap{});
}

gwn::gwn_status distance_any(ctx &c, dbuf<float> &x, dbuf<float> &y, dbuf<float> &z, dbuf<float> &o, float band) {
    if (c.bvh.accessor().internal_stack_bound <= 64)
        return distance_cfg<gwn::gwn_query_batch_config{256, 64}>(c, x, y, z, o, band);
    return distance_cfg<gwn::gwn_query_batch_config{256, 256}>(c, x, y, z, o, band);
}

template <gwn::gwn_query_batch_config Config>
gwn::gwn_status ray_cfg(ctx &c, dbuf<float> *r, dbuf<ray_result> &o, float t_min, float t_max) {
    return gwn::gwn_compute_ray_first_hit_batch<Config, 4, Real, Index, no_trap>(
        c.bvh, gwn::gwn_device_span<float const>(r[0].p, r[0].n), gwn::gwn_device_span<float const>(r[1].p, r[1].n),
        gwn::gwn_device_span<float const>(r[2].p, r[2].n), gwn::gwn_device_span<float const>(r[3].p, r[3].n),
        gwn::gwn_device_span<float const>(r[4].p, r[4].n), gwn::gwn_device_span<float const>(r[5].p, r[5].n),
        gwn::gwn_device_span<ray_result>(o.p, o.n), t_min, t_max, gwn::gwn_default_stream(), no_trap{});
}

gwn::gwn_status ray_any(ctx &c, dbuf<float> *r, dbuf<ray_result> &o, float t_min, float t_max) {
    if (c.bvh.accessor().internal_stack_bound <= 64)
        return ray_cfg<gwn::gwn_query_batch_config{256, 64}>(c, r, o, t_min, t_max);
    return ray_cfg<gwn::gwn_query_batch_config{256, 256}>(c, r, o, t_min, t_max);
}

// Mean device time (ms) of `iters` calls of run() after `warmup` untimed ones, each timed call
// bracketed by its own events on the legacy stream and preceded by a 256 MiB memset that flushes
// the L2 (126 MB on B200), as the library's own benchmark times its steps.
template <class F> int time_flushed(F &&run, int warmup, int iters, float *ms) {
    for (int i = 0; i < warmup; ++i) {
        auto s = run();
        if (!s.is_ok())
            return fail(s);
    }
    dbuf<unsigned char> flush(std::size_t(256) << 20);
    std::vector<cudaEvent_t> ev(2 * static_cast<std::size_t>(iters > 0 ? iters : 1));
    for (auto &e : ev)
        cudaEventCreate(&e);
    cudaDeviceSynchronize();
    for (int i = 0; i < iters; ++i) {
        cudaMemsetAsync(flush.p, i & 0xff, flush.n, cudaStreamLegacy);
        cudaEventRecord(ev[2 * i], cudaStreamLegacy);
        (void)run();
        cudaEventRecord(ev[2 * i + 1], cudaStreamLegacy);
    }
    cudaDeviceSynchronize();
    float total = 0;
    for (int i = 0; i < iters; ++i) {
        float t = 0;
        cudaEventElapsedTime(&t, ev[2 * i], ev[2 * i + 1]);
        total += t;
    }
    *ms = total / static_cast<float>(iters > 0 ? iters : 1);
    for (auto &e : ev)
        cudaEventDestroy(e);
    return static_cast<int>(cudaGetLastError());
}

} // namespace

extern "C" {

const char *ref_last_message(void) { return g_msg.c_str(); }

int ref_create(const float *x, const float *y, const float *z, uint64_t nv, const uint32_t *i0, const uint32_t *i1,
               const uint32_t *i2, uint64_t nt, void **out) {
    auto *c = new ctx{};
    auto s = gwn::gwn_upload_geometry(c->geometry, gwn::gwn_host_span<float const>(x, nv),
                                      gwn::gwn_host_span<float const>(y, nv), gwn::gwn_host_span<float const>(z, nv),
                                      gwn::gwn_host_span<Index const>(i0, nt), gwn::gwn_host_span<Index const>(i1, nt),
                                      gwn::gwn_host_span<Index const>(i2, nt));
    if (!s.is_ok()) {
        delete c;
        return fail(s);
    }
    *out = c;
    return 0;
}

void ref_destroy(void *p) {
    cudaDeviceSynchronize();
    delete static_cast<ctx *>(p);
}

int ref_build(void *p, int method, uint32_t radius, int morton_bits) {
    auto &c = *static_cast<ctx *>(p);
    gwn::gwn_bvh_build_options opt{};
    opt.method = method == 0 ? gwn::gwn_bvh_build_method::k_hploc : gwn::gwn_bvh_build_method::k_lbvh;
    opt.hploc_search_radius = radius;
    gwn::gwn_status s = morton_bits == 32 ? gwn::gwn_build_bvh<4, Real, Index, std::uint32_t>(c.geometry, c.bvh, opt)
                                          : gwn::gwn_build_bvh<4, Real, Index, std::uint64_t>(c.geometry, c.bvh, opt);
    return s.is_ok() ? 0 : fail(s);
}

// info: node_count, internal_stack_bound, packed_stack_bound, root reference, root bounds (6 floats)
int ref_bvh_info(void *p, uint64_t *node_count, uint32_t *ib, uint32_t *pb, uint64_t *root_ref, float *root_bounds) {
    auto const &a = static_cast<ctx *>(p)->bvh.accessor();
    *node_count = a.nodes.size();
    *ib = a.internal_stack_bound;
    *pb = a.packed_stack_bound;
    *root_ref = a.root.reference;
    std::memcpy(root_bounds, &a.root.bounds, 6 * sizeof(float));
    return 0;
}

int ref_bvh_copy(void *p, void *nodes, uint32_t *prims, void *tris) {
    auto const &a = static_cast<ctx *>(p)->bvh.accessor();
    cudaDeviceSynchronize();
    if (!a.nodes.empty())
        cudaMemcpy(nodes, a.nodes.data(), a.nodes.size_bytes(), cudaMemcpyDeviceToHost);
    cudaMemcpy(prims, a.primitive_indices.data(), a.primitive_indices.size_bytes(), cudaMemcpyDeviceToHost);
    cudaMemcpy(tris, a.triangles.data(), a.triangles.size_bytes(), cudaMemcpyDeviceToHost);
    return static_cast<int>(cudaGetLastError());
}

int ref_moment(void *p, int order) {
    auto &c = *static_cast<ctx *>(p);
    gwn::gwn_status s = order == 0   ? gwn::gwn_refit_bvh_moment<0>(c.bvh, c.m0)
                        : order == 1 ? gwn::gwn_refit_bvh_moment<1>(c.bvh, c.m1)
                                     : gwn::gwn_refit_bvh_moment<2>(c.bvh, c.m2);
    return s.is_ok() ? 0 : fail(s);
}

int ref_moment_copy(void *p, int order, void *host) {
    auto &c = *static_cast<ctx *>(p);
    cudaDeviceSynchronize();
    if (order == 0 && !c.m0.accessor().nodes.empty())
        cudaMemcpy(host, c.m0.accessor().nodes.data(), c.m0.accessor().nodes.size_bytes(), cudaMemcpyDeviceToHost);
    if (order == 1 && !c.m1.accessor().nodes.empty())
        cudaMemcpy(host, c.m1.accessor().nodes.data(), c.m1.accessor().nodes.size_bytes(), cudaMemcpyDeviceToHost);
    if (order == 2 && !c.m2.accessor().nodes.empty())
        cudaMemcpy(host, c.m2.accessor().nodes.data(), c.m2.accessor().nodes.size_bytes(), cudaMemcpyDeviceToHost);
    return static_cast<int>(cudaGetLastError());
}

int ref_exact(void *p, const float *qx, const float *qy, const float *qz, float *out, uint64_t n) {
    auto &c = *static_cast<ctx *>(p);
    dbuf<float> x(qx, n), y(qy, n), z(qz, n), o(n);
    auto s = gwn::gwn_compute_winding_number_exact_batch(
        c.bvh, gwn::gwn_device_span<float const>(x.p, n), gwn::gwn_device_span<float const>(y.p, n),
        gwn::gwn_device_span<float const>(z.p, n), gwn::gwn_device_span<float>(o.p, n));
    if (!s.is_ok())
        return fail(s);
    cudaDeviceSynchronize();
    o.to_host(out);
    return static_cast<int>(cudaGetLastError());
}

int ref_taylor(void *p, int order, const float *qx, const float *qy, const float *qz, float *out, uint64_t n,
               float beta) {
    auto &c = *static_cast<ctx *>(p);
    dbuf<float> x(qx, n), y(qy, n), z(qz, n), o(n);
    auto s = taylor_order(c, order, x, y, z, o, beta);
    if (!s.is_ok())
        return fail(s);
    cudaDeviceSynchronize();
    o.to_host(out);
    return static_cast<int>(cudaGetLastError());
}

// smallgwn's Taylor query gradient (gwn_compute_winding_gradient_taylor_batch) of a host batch.
int ref_taylor_gradient(void *p, int order, const float *qx, const float *qy, const float *qz, float *gx, float *gy,
                        float *gz, uint64_t n, float beta) {
    auto &c = *static_cast<ctx *>(p);
    if (c.bvh.accessor().internal_stack_bound > 64) {
        g_msg = "stack bound above 64";
        return -1;
    }
    dbuf<float> x(qx, n), y(qy, n), z(qz, n), ox(n), oy(n), oz(n);
    gwn::gwn_status s = order == 0   ? gradient_any<0>(c, c.m0, x, y, z, ox, oy, oz, beta)
                        : order == 1 ? gradient_any<1>(c, c.m1, x, y, z, ox, oy, oz, beta)
                                     : gradient_any<2>(c, c.m2, x, y, z, ox, oy, oz, beta);
    if (!s.is_ok())
        return fail(s);
    cudaDeviceSynchronize();
    ox.to_host(gx);
    oy.to_host(gy);
    oz.to_host(gz);
    return static_cast<int>(cudaGetLastError());
}

// Times `iters` Taylor batches (device-resident queries, L2 flushed before each) after `warmup`
// untimed ones; mean ms per batch. The moments of `order` must have been refit (ref_moment).
int ref_time_taylor(void *p, int order, const float *qx, const float *qy, const float *qz, uint64_t n, float beta,
                    int warmup, int iters, float *ms) {
    auto &c = *static_cast<ctx *>(p);
    dbuf<float> x(qx, n), y(qy, n), z(qz, n), o(n);
    return time_flushed([&]() { return taylor_order(c, order, x, y, z, o, beta); }, warmup, iters, ms);
}

int ref_time_exact(void *p, const float *qx, const float *qy, const float *qz, uint64_t n, int warmup, int iters,
                   float *ms) {
    auto &c = *static_cast<ctx *>(p);
    dbuf<float> x(qx, n), y(qy, n), z(qz, n), o(n);
    auto run = [&]() {
        return gwn::gwn_compute_winding_number_exact_batch(
            c.bvh, gwn::gwn_device_span<float const>(x.p, n), gwn::gwn_device_span<float const>(y.p, n),
            gwn::gwn_device_span<float const>(z.p, n), gwn::gwn_device_span<float>(o.p, n));
    };
    return time_flushed(run, warmup, iters, ms);
}

// Wall time of one gwn_build_bvh (host-synchronous by design in smallgwn), average over iters.
int ref_time_build(void *p, int method, uint32_t radius, int morton_bits, int iters, float *ms) {
    auto &c = *static_cast<ctx *>(p);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaDeviceSynchronize();
    cudaEventRecord(e0, cudaStreamLegacy);
    for (int i = 0; i < iters; ++i) {
        int rc = ref_build(p, method, radius, morton_bits);
        if (rc != 0)
            return rc;
    }
    cudaEventRecord(e1, cudaStreamLegacy);
    cudaEventSynchronize(e1);
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    *ms = t / static_cast<float>(iters > 0 ? iters : 1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    (void)c;
    return 0;
}

// Device time of one gwn_refit_bvh (order < 0) or gwn_refit_bvh_moment<order> on the built BVH,
// average over iters after one untimed call.
int ref_time_refit(void *p, int order, int iters, float *ms) {
    auto &c = *static_cast<ctx *>(p);
    auto run = [&]() -> int {
        if (order < 0) {
            auto s = gwn::gwn_refit_bvh(c.geometry, c.bvh);
            return s.is_ok() ? 0 : fail(s);
        }
        return ref_moment(p, order);
    };
    int rc = run();
    if (rc != 0)
        return rc;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaDeviceSynchronize();
    cudaEventRecord(e0, cudaStreamLegacy);
    for (int i = 0; i < iters && rc == 0; ++i)
        rc = run();
    cudaEventRecord(e1, cudaStreamLegacy);
    cudaEventSynchronize(e1);
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    *ms = t / static_cast<float>(iters > 0 ? iters : 1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}

int ref_update_refit(void *p, const float *x, const float *y, const float *z, uint64_t nv) {
    auto &c = *static_cast<ctx *>(p);
    auto s = gwn::gwn_update_geometry(c.geometry, gwn::gwn_host_span<float const>(x, nv),
                                      gwn::gwn_host_span<float const>(y, nv), gwn::gwn_host_span<float const>(z, nv));
    if (!s.is_ok())
        return fail(s);
    s = gwn::gwn_refit_bvh(c.geometry, c.bvh);
    return s.is_ok() ? 0 : fail(s);
}

// Uploads a query batch that ref_dynamic_frame evaluates on the device.
int ref_set_queries(void *p, const float *qx, const float *qy, const float *qz, uint64_t n) {
    auto &c = *static_cast<ctx *>(p);
    c.qx = std::make_unique<dbuf<float>>(qx, n);
    c.qy = std::make_unique<dbuf<float>>(qy, n);
    c.qz = std::make_unique<dbuf<float>>(qz, n);
    c.out = std::make_unique<dbuf<float>>(n);
    return static_cast<int>(cudaGetLastError());
}

// One frame of smallgwn's dynamic benchmark stage (tests/benchmark_main.cu:847-866): upload the
// frame's vertex positions from the host, refit the BVH, refit the moments of `order`, Taylor batch
// over the device-resident queries of ref_set_queries.
int ref_dynamic_frame(void *p, const float *x, const float *y, const float *z, uint64_t nv, int order, float beta) {
    auto &c = *static_cast<ctx *>(p);
    if (!c.qx)
        return 1;
    auto s = gwn::gwn_update_geometry(c.geometry, gwn::gwn_host_span<float const>(x, nv),
                                      gwn::gwn_host_span<float const>(y, nv), gwn::gwn_host_span<float const>(z, nv));
    if (!s.is_ok())
        return fail(s);
    s = gwn::gwn_refit_bvh(c.geometry, c.bvh);
    if (!s.is_ok())
        return fail(s);
    s = order == 0 ? gwn::gwn_refit_bvh_moment<0>(c.bvh, c.m0)
        : order == 1 ? gwn::gwn_refit_bvh_moment<1>(c.bvh, c.m1)
                     : gwn::gwn_refit_bvh_moment<2>(c.bvh, c.m2);
    if (!s.is_ok())
        return fail(s);
    s = taylor_order(c, order, *c.qx, *c.qy, *c.qz, *c.out, beta);
    return s.is_ok() ? 0 : fail(s);
}

// Build-stage outputs on the same geometry: sorted Morton codes (as uint64), sorted ids, sorted
// AABBs (6 floats each) -- gwn::detail::gwn_bvh_build_preprocess.
int ref_preprocess(void *p, int morton_bits, uint64_t *codes, uint32_t *ids, float *aabbs) {
    auto &c = *static_cast<ctx *>(p);
    std::size_t const n = c.geometry.triangle_count();
    try {
        if (morton_bits == 32) {
            gwn::detail::gwn_bvh_build_preprocess_data<Real, Index, std::uint32_t> pre{};
            gwn::detail::gwn_bvh_build_preprocess<std::uint32_t>(c.geometry.accessor(), pre, cudaStreamLegacy);
            cudaDeviceSynchronize();
            std::vector<std::uint32_t> h(n);
            cudaMemcpy(h.data(), pre.sorted_morton_codes.data(), n * 4, cudaMemcpyDeviceToHost);
            for (std::size_t i = 0; i < n; ++i)
                codes[i] = h[i];
            cudaMemcpy(ids, pre.sorted_primitive_indices.data(), n * 4, cudaMemcpyDeviceToHost);
            cudaMemcpy(aabbs, pre.sorted_primitive_aabbs.data(), n * 24, cudaMemcpyDeviceToHost);
        } else {
            gwn::detail::gwn_bvh_build_preprocess_data<Real, Index, std::uint64_t> pre{};
            gwn::detail::gwn_bvh_build_preprocess<std::uint64_t>(c.geometry.accessor(), pre, cudaStreamLegacy);
            cudaDeviceSynchronize();
            cudaMemcpy(codes, pre.sorted_morton_codes.data(), n * 8, cudaMemcpyDeviceToHost);
            cudaMemcpy(ids, pre.sorted_primitive_indices.data(), n * 4, cudaMemcpyDeviceToHost);
            cudaMemcpy(aabbs, pre.sorted_primitive_aabbs.data(), n * 24, cudaMemcpyDeviceToHost);
        }
    } catch (std::exception const &e) {
        g_msg = e.what();
        return 3;
    }
    return static_cast<int>(cudaGetLastError());
}

// Binary LBVH / H-PLOC on host sorted codes (uint64 storage) and AABBs. nodes: 4 uint32 per
// internal node (left index, left kind, right index, right kind); bounds: 6 floats per node.
int ref_binary(int method, int morton_bits, uint64_t n, const uint64_t *codes, const float *aabbs, uint32_t radius,
               uint32_t *nodes, float *bounds, uint32_t *root) {
    try {
        dbuf<gwn::gwn_aabb<Real>> d_aabb(reinterpret_cast<gwn::gwn_aabb<Real> const *>(aabbs), n);
        gwn::detail::gwn_device_array<gwn::detail::gwn_binary_node<Index>> bn{};
        gwn::detail::gwn_device_array<Index> parent{};
        gwn::detail::gwn_device_array<gwn::gwn_aabb<Real>> bb{};
        Index r = 0;
        auto run = [&](auto const *dcodes, auto tag) {
            using MC = decltype(tag);
            cuda::std::span<MC const> cs(dcodes, n);
            cuda::std::span<gwn::gwn_aabb<Real> const> as(d_aabb.p, n);
            if (method == 1) {
                gwn::detail::gwn_bvh_build_binary_lbvh<Real, Index, MC>(cs, as, bn, parent, bb, cudaStreamLegacy);
                r = 0;
            } else {
                dbuf<Index> ids(n);
                gwn::detail::gwn_bvh_build_binary_hploc_impl<Real, Index, MC>(
                    cuda::std::span<Index const>(ids.p, n), cs, as, bn, parent, bb, r, radius, cudaStreamLegacy);
            }
        };
        if (morton_bits == 32) {
            std::vector<std::uint32_t> h(n);
            for (std::size_t i = 0; i < n; ++i)
                h[i] = static_cast<std::uint32_t>(codes[i]);
            dbuf<std::uint32_t> dc(h.data(), n);
            run(dc.p, std::uint32_t{});
        } else {
            dbuf<std::uint64_t> dc(codes, n);
            run(dc.p, std::uint64_t{});
        }
        cudaDeviceSynchronize();
        std::vector<gwn::detail::gwn_binary_node<Index>> hn(n - 1);
        cudaMemcpy(hn.data(), bn.data(), (n - 1) * sizeof(hn[0]), cudaMemcpyDeviceToHost);
        for (std::size_t i = 0; i + 1 < n; ++i) {
            nodes[4 * i + 0] = hn[i].left.index;
            nodes[4 * i + 1] = hn[i].left.kind;
            nodes[4 * i + 2] = hn[i].right.index;
            nodes[4 * i + 3] = hn[i].right.kind;
        }
        cudaMemcpy(bounds, bb.data(), (n - 1) * 24, cudaMemcpyDeviceToHost);
        *root = r;
    } catch (std::exception const &e) {
        g_msg = e.what();
        return 3;
    }
    return static_cast<int>(cudaGetLastError());
}

// FP64 exact winding (the Real = double instantiation), LBVH build, host arrays.
int ref_exact_f64(const double *x, const double *y, const double *z, uint64_t nv, const uint32_t *i0,
                  const uint32_t *i1, const uint32_t *i2, uint64_t nt, const double *qx, const double *qy,
                  const double *qz, double *out, uint64_t n) {
    gwn::gwn_geometry_object<double, Index> g;
    auto s = gwn::gwn_upload_geometry(g, gwn::gwn_host_span<double const>(x, nv), gwn::gwn_host_span<double const>(y, nv),
                                      gwn::gwn_host_span<double const>(z, nv), gwn::gwn_host_span<Index const>(i0, nt),
                                      gwn::gwn_host_span<Index const>(i1, nt), gwn::gwn_host_span<Index const>(i2, nt));
    if (!s.is_ok())
        return fail(s);
    gwn::gwn_bvh4_object<double, Index> b;
    gwn::gwn_bvh_build_options opt{};
    opt.method = gwn::gwn_bvh_build_method::k_lbvh;
    s = gwn::gwn_build_bvh(g, b, opt);
    if (!s.is_ok())
        return fail(s);
    dbuf<double> dx(qx, n), dy(qy, n), dz(qz, n), o(n);
    s = gwn::gwn_compute_winding_number_exact_batch(b, gwn::gwn_device_span<double const>(dx.p, n),
                                                    gwn::gwn_device_span<double const>(dy.p, n),
                                                    gwn::gwn_device_span<double const>(dz.p, n),
                                                    gwn::gwn_device_span<double>(o.p, n));
    if (!s.is_ok())
        return fail(s);
    cudaDeviceSynchronize();
    o.to_host(out);
    return static_cast<int>(cudaGetLastError());
}

// smallgwn's unsigned-distance batch (gwn_compute_unsigned_distance_batch) of a host batch.
int ref_distance(void *p, const float *qx, const float *qy, const float *qz, float *out, uint64_t n, float band) {
    auto &c = *static_cast<ctx *>(p);
    dbuf<float> x(qx, n), y(qy, n), z(qz, n), o(n);
    auto s = distance_any(c, x, y, z, o, band);
    if (!s.is_ok())
        return fail(s);
    cudaDeviceSynchronize();
    o.to_host(out);
    return static_cast<int>(cudaGetLastError());
}

// smallgwn's ray first-hit batch (gwn_compute_ray_first_hit_batch) of a host batch; `out` receives
// n 32-byte gwn_ray_first_hit_result records.
int ref_ray(void *p, const float *ox, const float *oy, const float *oz, const float *dx, const float *dy,
            const float *dz, void *out, uint64_t n, float t_min, float t_max) {
    auto &c = *static_cast<ctx *>(p);
    dbuf<float> r[6] = {dbuf<float>(ox, n), dbuf<float>(oy, n), dbuf<float>(oz, n),
                        dbuf<float>(dx, n), dbuf<float>(dy, n), dbuf<float>(dz, n)};
    dbuf<ray_result> o(n);
    auto s = ray_any(c, r, o, t_min, t_max);
    if (!s.is_ok())
        return fail(s);
    cudaDeviceSynchronize();
    o.to_host(static_cast<ray_result *>(out));
    return static_cast<int>(cudaGetLastError());
}

// Times `iters` distance (kind 0) or ray (kind 1) batches on device-resident inputs after `warmup`
// untimed ones; average ms per batch.
int ref_time_spatial(void *p, int kind, const float *qx, const float *qy, const float *qz, const float *dx,
                     const float *dy, const float *dz, uint64_t n, float band, float t_min, float t_max, int warmup,
                     int iters, float *ms) {
    auto &c = *static_cast<ctx *>(p);
    dbuf<float> r[6] = {dbuf<float>(qx, n), dbuf<float>(qy, n), dbuf<float>(qz, n),
                        dbuf<float>(kind ? dx : qx, n), dbuf<float>(kind ? dy : qy, n), dbuf<float>(kind ? dz : qz, n)};
    dbuf<float> od(kind ? 0 : n);
    dbuf<ray_result> orr(kind ? n : 0);
    auto run = [&]() { return kind ? ray_any(c, r, orr, t_min, t_max) : distance_any(c, r[0], r[1], r[2], od, band); };
    for (int i = 0; i < warmup; ++i) {
        auto s = run();
        if (!s.is_ok())
            return fail(s);
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaDeviceSynchronize();
    cudaEventRecord(e0, cudaStreamLegacy);
    for (int i = 0; i < iters; ++i)
        (void)run();
    cudaEventRecord(e1, cudaStreamLegacy);
    cudaEventSynchronize(e1);
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    *ms = t / static_cast<float>(iters > 0 ? iters : 1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return static_cast<int>(cudaGetLastError());
}

// smallgwn's boundary chain of the context's geometry (gwn_build_boundary_chain). With start ==
// nullptr only builds and reports the row count.
int ref_boundary(void *p, uint32_t *start, uint32_t *end, uint64_t *mult, uint64_t *count) {
    auto &c = *static_cast<ctx *>(p);
    auto s = gwn::gwn_build_boundary_chain(c.geometry, c.chain);
    if (!s.is_ok())
        return fail(s);
    cudaDeviceSynchronize();
    auto const &a = c.chain.accessor();
    *count = a.edge_count();
    if (start != nullptr && a.edge_count() > 0) {
        cudaMemcpy(start, a.start_vertex.data(), a.edge_count() * sizeof(uint32_t), cudaMemcpyDeviceToHost);
        cudaMemcpy(end, a.end_vertex.data(), a.edge_count() * sizeof(uint32_t), cudaMemcpyDeviceToHost);
        cudaMemcpy(mult, a.multiplicity.data(), a.edge_count() * sizeof(uint64_t), cudaMemcpyDeviceToHost);
    }
    return static_cast<int>(cudaGetLastError());
}

// smallgwn's antipodal winding batch (needs ref_build and ref_boundary first).
int ref_antipodal(void *p, const float *qx, const float *qy, const float *qz, float *out, uint64_t n) {
    auto &c = *static_cast<ctx *>(p);
    dbuf<float> x(qx, n), y(qy, n), z(qz, n), o(n);
    gwn::gwn_status s;
    if (c.bvh.accessor().internal_stack_bound <= 64)
        s = gwn::gwn_compute_winding_number_antipodal_batch<gwn::gwn_query_batch_config{256, 64}, 4, Real, Index, no_trap>(
            c.geometry, c.bvh, c.chain, gwn::gwn_device_span<float const>(x.p, n), gwn::gwn_device_span<float const>(y.p, n),
            gwn::gwn_device_span<float const>(z.p, n), gwn::gwn_device_span<float>(o.p, n), gwn::gwn_default_stream(),
            no_trap{});
    else
        s = gwn::gwn_compute_winding_number_antipodal_batch<gwn::gwn_query_batch_config{256, 256}, 4, Real, Index, no_trap>(
            c.geometry, c.bvh, c.chain, gwn::gwn_device_span<float const>(x.p, n), gwn::gwn_device_span<float const>(y.p, n),
            gwn::gwn_device_span<float const>(z.p, n), gwn::gwn_device_span<float>(o.p, n), gwn::gwn_default_stream(),
            no_trap{});
    if (!s.is_ok())
        return fail(s);
    cudaDeviceSynchronize();
    o.to_host(out);
    return static_cast<int>(cudaGetLastError());
}

// smallgwn's antipodal gradient batch (needs ref_boundary first).
int ref_antipodal_gradient(void *p, const float *qx, const float *qy, const float *qz, float *gx, float *gy, float *gz,
                           uint64_t n) {
    auto &c = *static_cast<ctx *>(p);
    dbuf<float> x(qx, n), y(qy, n), z(qz, n), ox(n), oy(n), oz(n);
    auto s = gwn::gwn_compute_winding_gradient_antipodal_batch(
        c.geometry, c.chain, gwn::gwn_device_span<float const>(x.p, n), gwn::gwn_device_span<float const>(y.p, n),
        gwn::gwn_device_span<float const>(z.p, n), gwn::gwn_device_span<float>(ox.p, n),
        gwn::gwn_device_span<float>(oy.p, n), gwn::gwn_device_span<float>(oz.p, n));
    if (!s.is_ok())
        return fail(s);
    cudaDeviceSynchronize();
    ox.to_host(gx);
    oy.to_host(gy);
    oz.to_host(gz);
    return static_cast<int>(cudaGetLastError());
}

// Average ms of `iters` antipodal batches on device-resident queries after `warmup` untimed ones.
int ref_time_antipodal(void *p, const float *qx, const float *qy, const float *qz, uint64_t n, int warmup, int iters,
                       float *ms) {
    auto &c = *static_cast<ctx *>(p);
    dbuf<float> x(qx, n), y(qy, n), z(qz, n), o(n);
    auto run = [&]() {
        return gwn::gwn_compute_winding_number_antipodal_batch<gwn::gwn_query_batch_config{256, 64}, 4, Real, Index,
                                                               no_trap>(
            c.geometry, c.bvh, c.chain, gwn::gwn_device_span<float const>(x.p, n), gwn::gwn_device_span<float const>(y.p, n),
            gwn::gwn_device_span<float const>(z.p, n), gwn::gwn_device_span<float>(o.p, n), gwn::gwn_default_stream(),
            no_trap{});
    };
    for (int i = 0; i < warmup; ++i) {
        auto s = run();
        if (!s.is_ok())
            return fail(s);
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaDeviceSynchronize();
    cudaEventRecord(e0, cudaStreamLegacy);
    for (int i = 0; i < iters; ++i)
        (void)run();
    cudaEventRecord(e1, cudaStreamLegacy);
    cudaEventSynchronize(e1);
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    *ms = t / static_cast<float>(iters > 0 ? iters : 1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return static_cast<int>(cudaGetLastError());
}

} // extern "C"
