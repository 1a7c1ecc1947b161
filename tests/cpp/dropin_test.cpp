// Drop-in API test: smallgwn-style C++ code (include/gwn/gwn.cuh) compiled by a plain C++20 host
// compiler and linked against libgwnb.so. Each case restates one of smallgwn's unit tests:
//   leaf-root build record          tests/unit_gwn_bvh.cu:93-139
//   two-triangle query records      tests/unit_gwn_bvh.cu:141-218
//   refit bounds and primitive order tests/unit_gwn_bvh.cu:220-287
//   rejected options keep the BVH   tests/unit_gwn_bvh.cu:289-358
//   exact vs CPU, asymmetric octahedron  tests/unit_gwn_query_winding.cu:193-215
//   full-descent Taylor == exact    tests/unit_gwn_bvh_moment.cu:42-114
//   stale moments are rejected      tests/unit_gwn_bvh_moment.cu:116-156
//   distance and ray on 12 layers   tests/unit_gwn_query_distance_ray.cu:361-396
//   open-cube boundary, antipodal   tests/unit_gwn_boundary.cu:125-150, tests/unit_gwn_query_antipodal.cu:368-381
//   matrix upload (Eigen bridge)    include/gwn/gwn_eigen_bridge.cuh:26-132
//   PLY meshes, scene files         tests/test_mesh_io.cpp:43-92 (scene files have no counterpart)
// Exit code 0 when every check passes; `--compile-only` exits before touching the GPU and
// `--host-checks` runs only the cases that need no GPU.
#include <gwn/gwn.cuh>
#include <gwn/gwn_eigen_bridge.cuh>

#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <limits>
#include <string>
#include <unistd.h>
#include <vector>

namespace {

int g_failures = 0;

#define CHECK(cond)                                                                                \
    do {                                                                                           \
        if (!(cond)) {                                                                             \
            std::fprintf(stderr, "%s:%d: CHECK failed: %s\n", __FILE__, __LINE__, #cond);          \
            ++g_failures;                                                                          \
        }                                                                                          \
    } while (0)

using Real = float;
using Index = std::uint32_t;

template <class T> gwn::gwn_host_span<T const> hs(std::vector<T> const &v) { return {v.data(), v.size()}; }
template <class T, std::size_t N> gwn::gwn_host_span<T const> hs(std::array<T, N> const &v) {
    return {v.data(), v.size()};
}

struct dbuf {
    float *p = nullptr;
    std::size_t n = 0;
    explicit dbuf(std::vector<float> const &h) : n(h.size()) {
        cudaMalloc(&p, n * sizeof(float));
        cudaMemcpy(p, h.data(), n * sizeof(float), cudaMemcpyHostToDevice);
    }
    explicit dbuf(std::size_t count) : n(count) { cudaMalloc(&p, n * sizeof(float)); }
    ~dbuf() { cudaFree(p); }
    std::vector<float> host() const {
        std::vector<float> h(n);
        cudaDeviceSynchronize();
        cudaMemcpy(h.data(), p, n * sizeof(float), cudaMemcpyDeviceToHost);
        return h;
    }
    gwn::gwn_device_span<float const> in() const { return {p, n}; }
    gwn::gwn_device_span<float> out() { return {p, n}; }
};

template <class T> std::vector<T> to_host(cuda::std::span<T> s) {
    std::vector<T> h(s.size());
    cudaDeviceSynchronize();
    cudaMemcpy(h.data(), s.data(), s.size_bytes(), cudaMemcpyDeviceToHost);
    return h;
}

double cpu_winding(std::vector<float> const &x, std::vector<float> const &y, std::vector<float> const &z,
                   std::vector<Index> const &i0, std::vector<Index> const &i1, std::vector<Index> const &i2,
                   double qx, double qy, double qz) {
    double sum = 0;
    for (std::size_t t = 0; t < i0.size(); ++t) {
        double a[3] = {x[i0[t]] - qx, y[i0[t]] - qy, z[i0[t]] - qz};
        double b[3] = {x[i1[t]] - qx, y[i1[t]] - qy, z[i1[t]] - qz};
        double c[3] = {x[i2[t]] - qx, y[i2[t]] - qy, z[i2[t]] - qz};
        double la = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
        double lb = std::sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
        double lc = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
        double num = a[0] * (b[1] * c[2] - b[2] * c[1]) + a[1] * (b[2] * c[0] - b[0] * c[2]) +
                     a[2] * (b[0] * c[1] - b[1] * c[0]);
        double den = la * lb * lc + (a[0] * b[0] + a[1] * b[1] + a[2] * b[2]) * lc +
                     (a[0] * c[0] + a[1] * c[1] + a[2] * c[2]) * lb + (b[0] * c[0] + b[1] * c[1] + b[2] * c[2]) * la;
        sum += 2 * std::atan2(num, den);
    }
    return sum / (4 * M_PI);
}

void leaf_root_build() {
    std::vector<float> x{0, 1, 0}, y{0, 0, 1}, z{0, 0, 0};
    std::vector<Index> i0{0}, i1{1}, i2{2};
    gwn::gwn_geometry_object<Real, Index> geometry;
    CHECK(gwn::gwn_upload_geometry(geometry, hs(x), hs(y), hs(z), hs(i0), hs(i1), hs(i2)).is_ok());
    gwn::gwn_bvh4_object<Real, Index> bvh;
    CHECK(gwn::gwn_build_bvh(geometry, bvh).is_ok());
    auto const &a = bvh.accessor();
    CHECK(a.is_valid() && a.has_leaf_root() && a.nodes.empty());
    CHECK(a.root.offset() == 0 && a.root.primitive_count() == 1);
    CHECK(a.root.bounds.min_x == 0 && a.root.bounds.max_x == 1 && a.root.bounds.max_y == 1 && a.root.bounds.max_z == 0);
    auto tris = to_host(a.triangles);
    CHECK(tris.size() == 1 && tris[0].e1_x == 1 && tris[0].e2_y == 1 && tris[0].v0_z == 0);
}

void two_triangle_records_and_refit() {
    std::vector<float> x{0, 1, 0, 4, 6, 4}, y{0, 0, 2, 0, 0, 3}, z{1, 1, 1, -2, -2, -2};
    std::vector<Index> i0{0, 3}, i1{1, 4}, i2{2, 5};
    gwn::gwn_geometry_object<Real, Index> geometry;
    CHECK(gwn::gwn_upload_geometry(geometry, hs(x), hs(y), hs(z), hs(i0), hs(i1), hs(i2)).is_ok());
    gwn::gwn_bvh4_object<Real, Index> bvh;
    CHECK(gwn::gwn_build_bvh(geometry, bvh, gwn::gwn_bvh_build_options{.method = gwn::gwn_bvh_build_method::k_lbvh})
              .is_ok());
    CHECK(bvh.accessor().nodes.size() == 1 && bvh.accessor().root.is_internal());
    auto nodes = to_host(bvh.accessor().nodes);
    int leaves = 0;
    for (int s = 0; s < 4; ++s)
        leaves += nodes[0].child(s).is_leaf() ? 1 : 0;
    CHECK(leaves == 2);
    auto order = to_host(bvh.accessor().primitive_indices);

    x = {-7, -2, -7, 8, 11, 8};
    y = {5, 5, 9, -4, -4, 2};
    z = {3, 3, 3, -6, -6, -6};
    CHECK(gwn::gwn_update_geometry(geometry, hs(x), hs(y), hs(z)).is_ok());
    CHECK(gwn::gwn_refit_bvh(geometry, bvh).is_ok());
    auto const &a = bvh.accessor();
    CHECK(to_host(a.primitive_indices) == order);
    CHECK(a.root.bounds.min_x == -7 && a.root.bounds.min_y == -4 && a.root.bounds.min_z == -6);
    CHECK(a.root.bounds.max_x == 11 && a.root.bounds.max_y == 9 && a.root.bounds.max_z == 3);
    auto tris = to_host(a.triangles);
    for (std::size_t s = 0; s < tris.size(); ++s) {
        Index const p = order[s];
        CHECK(tris[s].v0_x == x[i0[p]] && tris[s].e1_y == y[i1[p]] - y[i0[p]] && tris[s].e2_z == z[i2[p]] - z[i0[p]]);
    }
}

void rejected_options_keep_bvh() {
    std::vector<float> x{0, 1, 0}, y{0, 0, 1}, z{0, 0, 0};
    std::vector<Index> i0{0}, i1{1}, i2{2};
    gwn::gwn_geometry_object<Real, Index> geometry;
    CHECK(gwn::gwn_upload_geometry(geometry, hs(x), hs(y), hs(z), hs(i0), hs(i1), hs(i2)).is_ok());
    gwn::gwn_bvh4_object<Real, Index> bvh;
    CHECK(gwn::gwn_build_bvh(geometry, bvh).is_ok());
    auto *prims = bvh.accessor().primitive_indices.data();
    for (std::uint32_t r : {0u, 9u}) {
        auto st = gwn::gwn_build_bvh(geometry, bvh, gwn::gwn_bvh_build_options{gwn::gwn_bvh_build_method::k_hploc, r});
        CHECK(st.error() == gwn::gwn_error::invalid_argument);
        CHECK(bvh.accessor().primitive_indices.data() == prims && bvh.has_data());
    }
    gwn::gwn_geometry_object<double, Index> dgeo;
    std::vector<double> dx{0, 1, 0};
    auto st = gwn::gwn_upload_geometry(dgeo, hs(dx), hs(dx), hs(dx), hs(i0), hs(i1), hs(i2));
    CHECK(st.error() == gwn::gwn_error::invalid_argument);
}

void queries_match_cpu() {
    std::vector<float> x{1.7f, -0.8f, 0.15f, -0.1f, 0.2f, -0.2f}, y{0.1f, -0.2f, 1.2f, -0.7f, 0.1f, -0.1f},
        z{0, 0.1f, -0.1f, 0.15f, 1.5f, -0.9f};
    std::vector<Index> i0{0, 2, 1, 3, 2, 1, 3, 0}, i1{2, 1, 3, 0, 0, 2, 1, 3}, i2{4, 4, 4, 4, 5, 5, 5, 5};
    gwn::gwn_geometry_object<Real, Index> geometry;
    CHECK(gwn::gwn_upload_geometry(geometry, hs(x), hs(y), hs(z), hs(i0), hs(i1), hs(i2)).is_ok());
    gwn::gwn_bvh4_object<Real, Index> bvh;
    CHECK(gwn::gwn_build_bvh(geometry, bvh).is_ok());
    std::vector<float> qx{0, 4, -2, 0.2f, 1.5f}, qy{0, 3, 1, -1.4f, 0.2f}, qz{0, 2, -3, 2.2f, -1.8f};
    dbuf dx(qx), dy(qy), dz(qz), exact(qx.size()), taylor(qx.size());
    CHECK(gwn::gwn_compute_winding_number_exact_batch(bvh, dx.in(), dy.in(), dz.in(), exact.out()).is_ok());
    gwn::gwn_bvh4_moment_object<1, Real, Index> moment;
    CHECK(gwn::gwn_refit_bvh_moment<1>(bvh, moment).is_ok());
    CHECK(moment.accessor().is_valid_for(bvh.accessor()));
    CHECK(gwn::gwn_compute_winding_number_taylor_batch<1>(bvh, moment, dx.in(), dy.in(), dz.in(), taylor.out(),
                                                          Real(1e6))
              .is_ok());
    auto he = exact.host();
    auto ht = taylor.host();
    for (std::size_t i = 0; i < qx.size(); ++i) {
        double const ref = cpu_winding(x, y, z, i0, i1, i2, qx[i], qy[i], qz[i]);
        CHECK(std::abs(he[i] - ref) <= 1e-5);
        CHECK(std::abs(ht[i] - he[i]) <= 1e-6);
    }
    // smallgwn accepts batch block sizes up to 1024: the same results with 512- and 1024-thread configs
    constexpr gwn::gwn_query_batch_config k_wide{512, 64};
    constexpr gwn::gwn_query_batch_config k_widest{1024, 64};
    dbuf wide(qx.size()), widest(qx.size());
    CHECK((gwn::gwn_compute_winding_number_taylor_batch<1, k_wide>(bvh, moment, dx.in(), dy.in(), dz.in(),
                                                                   wide.out(), Real(1e6))
               .is_ok()));
    CHECK((gwn::gwn_compute_winding_number_taylor_batch<1, k_widest>(bvh, moment, dx.in(), dy.in(), dz.in(),
                                                                     widest.out(), Real(1e6))
               .is_ok()));
    auto hw = wide.host();
    auto hww = widest.host();
    for (std::size_t i = 0; i < qx.size(); ++i)
        CHECK(hw[i] == ht[i] && hww[i] == ht[i]);
    // a refit publishes a new revision: the old moments are stale
    CHECK(gwn::gwn_refit_bvh(geometry, bvh).is_ok());
    CHECK(!moment.accessor().is_valid_for(bvh.accessor()));
    auto st = gwn::gwn_compute_winding_number_taylor_batch<1>(bvh, moment, dx.in(), dy.in(), dz.in(), taylor.out());
    CHECK(st.error() == gwn::gwn_error::invalid_argument);
    // stack capacity below the BVH's bound is rejected up front
    constexpr gwn::gwn_query_batch_config k_tiny{256, 1};
    CHECK(gwn::gwn_refit_bvh_moment<1>(bvh, moment).is_ok());
    if (bvh.accessor().internal_stack_bound > 1) {
        st = gwn::gwn_compute_winding_number_taylor_batch<1, k_tiny>(bvh, moment, dx.in(), dy.in(), dz.in(),
                                                                     taylor.out());
        CHECK(st.error() == gwn::gwn_error::invalid_argument);
        CHECK(st.message().find("Traversal stack capacity") != std::string::npos);
    }
}

void distance_and_ray_on_layers() {
    std::vector<float> x, y, z;
    std::vector<Index> i0, i1, i2;
    for (Index t = 0; t < 12; ++t) {
        Index const v = static_cast<Index>(x.size());
        x.insert(x.end(), {0, 1, 0});
        y.insert(y.end(), {0, 0, 1});
        z.insert(z.end(), {float(t), float(t), float(t)});
        i0.push_back(v);
        i1.push_back(v + 1);
        i2.push_back(v + 2);
    }
    gwn::gwn_geometry_object<Real, Index> geometry;
    CHECK(gwn::gwn_upload_geometry(geometry, hs(x), hs(y), hs(z), hs(i0), hs(i1), hs(i2)).is_ok());
    gwn::gwn_bvh4_object<Real, Index> bvh;
    CHECK(gwn::gwn_build_bvh(geometry, bvh).is_ok());
    dbuf ox(std::vector<float>{0.25f, 2, 0}), oy(std::vector<float>{0.25f, 2, 0.25f}), oz(std::vector<float>{20, 20, 20});
    dbuf dx(std::vector<float>{0, 0, 0}), dy(std::vector<float>{0, 0, 0}), dz(std::vector<float>{-1, -1, -1});
    gwn::gwn_ray_first_hit_result<Real, Index> *hits = nullptr;
    cudaMalloc(&hits, 3 * sizeof(*hits));
    CHECK(gwn::gwn_compute_ray_first_hit_batch(bvh, ox.in(), oy.in(), oz.in(), dx.in(), dy.in(), dz.in(),
                                               gwn::gwn_device_span<gwn::gwn_ray_first_hit_result<Real, Index>>(hits, 3))
              .is_ok());
    std::vector<gwn::gwn_ray_first_hit_result<Real, Index>> h(3);
    cudaDeviceSynchronize();
    cudaMemcpy(h.data(), hits, 3 * sizeof(*hits), cudaMemcpyDeviceToHost);
    cudaFree(hits);
    CHECK(h[0].hit() && h[0].t == 9 && h[0].primitive_id == 11);
    CHECK(!h[1].hit() && h[1].t == -1 && h[1].primitive_id == gwn::gwn_invalid_index<Index>());
    CHECK(h[2].hit() && h[2].t == 9 && h[2].primitive_id == 11);
    dbuf qx(std::vector<float>{0.25f, 0.25f, 0}), qy(std::vector<float>{0.25f, 0.25f, 0.25f}),
        qz(std::vector<float>{10.25f, 30, 10.25f}), d(3);
    CHECK(gwn::gwn_compute_unsigned_distance_batch(bvh, qx.in(), qy.in(), qz.in(), d.out(), Real(2)).is_ok());
    auto hd = d.host();
    CHECK(hd[0] == 0.25f && hd[1] == 2 && hd[2] == 0.25f);
}

void open_cube_boundary_and_antipodal() {
    std::vector<float> x{-1, 1, 1, -1, -1, 1, 1, -1}, y{-1, -1, 1, 1, -1, -1, 1, 1}, z{-1, -1, -1, -1, 1, 1, 1, 1};
    std::vector<Index> i0{0, 0, 0, 0, 1, 1, 0, 0, 3, 3}, i1{2, 3, 4, 7, 2, 6, 1, 5, 7, 6}, i2{1, 2, 7, 3, 6, 5, 5, 4, 6, 2};
    gwn::gwn_geometry_object<Real, Index> geometry;
    CHECK(gwn::gwn_upload_geometry(geometry, hs(x), hs(y), hs(z), hs(i0), hs(i1), hs(i2)).is_ok());
    gwn::gwn_boundary_chain_object<Index> chain;
    CHECK(gwn::gwn_build_boundary_chain(geometry, chain).is_ok());
    CHECK(chain.has_data() && chain.accessor().edge_count() == 4);
    auto st = to_host(chain.accessor().start_vertex);
    auto en = to_host(chain.accessor().end_vertex);
    auto mu = to_host(chain.accessor().multiplicity);
    int found = 0;
    for (std::size_t i = 0; i < st.size(); ++i)
        for (auto [a, b] : {std::pair<Index, Index>{4, 7}, {5, 4}, {6, 5}, {7, 6}})
            found += (st[i] == a && en[i] == b && mu[i] == 1) ? 1 : 0;
    CHECK(found == 4);
    gwn::gwn_bvh4_object<Real, Index> bvh;
    CHECK(gwn::gwn_build_bvh(geometry, bvh).is_ok());
    std::vector<float> qx{0.23f, 2.2f, -0.41f, -2.3f}, qy{0.17f, 0.3f, 0.26f, -0.4f}, qz{0.11f, 0.2f, 1.7f, 0.5f};
    dbuf dx(qx), dy(qy), dz(qz), w(qx.size()), gx(qx.size()), gy(qx.size()), gz(qx.size());
    CHECK(gwn::gwn_compute_winding_number_antipodal_batch(geometry, bvh, chain, dx.in(), dy.in(), dz.in(), w.out())
              .is_ok());
    CHECK(gwn::gwn_compute_winding_gradient_antipodal_batch(geometry, chain, dx.in(), dy.in(), dz.in(), gx.out(),
                                                            gy.out(), gz.out())
              .is_ok());
    auto hw = w.host();
    auto hg = gx.host();
    for (std::size_t i = 0; i < qx.size(); ++i) {
        CHECK(std::abs(hw[i] - cpu_winding(x, y, z, i0, i1, i2, qx[i], qy[i], qz[i])) <= 3e-4);
        CHECK(std::isfinite(hg[i]));
    }
    gwn::gwn_boundary_chain_object<Index> missing;
    CHECK(gwn::gwn_compute_winding_number_antipodal_batch(geometry, bvh, missing, dx.in(), dy.in(), dz.in(), w.out())
              .error() == gwn::gwn_error::invalid_argument);
}


/// Row- or column-major dense matrix with Eigen's element interface (rows(), cols(), (r, c)).
template <class T, bool RowMajor> struct fake_matrix {
    long r = 0, c = 0;
    std::vector<T> data;
    fake_matrix(long rows, long cols, std::vector<T> row_major) : r(rows), c(cols), data(rows * cols) {
        for (long i = 0; i < rows; ++i)
            for (long j = 0; j < cols; ++j)
                (*this)(i, j) = row_major[i * cols + j];
    }
    long rows() const { return r; }
    long cols() const { return c; }
    T &operator()(long i, long j) { return RowMajor ? data[i * c + j] : data[j * r + i]; }
    T const &operator()(long i, long j) const { return RowMajor ? data[i * c + j] : data[j * r + i]; }
};

std::vector<double> const k_cube_v{-1, -1, -1, 1, -1, -1, 1, 1, -1, -1, 1, -1, -1, -1, 1, 1, -1, 1, 1, 1, 1, -1, 1, 1};
std::vector<int> const k_cube_f{0, 2, 1, 0, 3, 2, 4, 5, 6, 4, 6, 7, 0, 1, 5, 0, 5, 4,
                                3, 7, 6, 3, 6, 2, 0, 4, 7, 0, 7, 3, 1, 2, 6, 1, 6, 5};

std::filesystem::path scratch(char const *name) {
    return std::filesystem::temp_directory_path() / (std::string("gwnb_dropin_") + std::to_string(getpid()) + "_" + name);
}

void eigen_bridge_refusals() {
    gwn::gwn_geometry_object<Real, Index> geometry;
    fake_matrix<double, true> v(8, 3, k_cube_v);
    fake_matrix<double, true> v2(4, 2, std::vector<double>(8, 0.0));
    fake_matrix<int, false> f(12, 3, k_cube_f);
    auto st = gwn::gwn_upload_geometry_from_eigen(geometry, v2, f);
    CHECK(st.error() == gwn::gwn_error::invalid_argument && st.message().find("Nx3") != std::string::npos);
    for (double bad : {-1.0, 8.0, 1.5, std::numeric_limits<double>::quiet_NaN(), 1e30}) {
        std::vector<double> fv(k_cube_f.begin(), k_cube_f.end());
        fv[7] = bad;
        fake_matrix<double, true> fd(12, 3, fv);
        st = gwn::gwn_upload_geometry_from_eigen(geometry, v, fd);
        CHECK(st.error() == gwn::gwn_error::invalid_argument &&
              st.message().find("integer-valued") != std::string::npos);
    }
    std::vector<int> fi = k_cube_f;
    fi[35] = -3;
    st = gwn::gwn_upload_geometry_from_eigen(geometry, v, fake_matrix<int, false>(12, 3, fi));
    CHECK(st.error() == gwn::gwn_error::invalid_argument);
    CHECK(!geometry.has_data());
}

void ply_round_trip_on_host() {
    gwn::gwn_host_mesh mesh;
    for (std::size_t i = 0; i < 8; ++i) {
        mesh.vertex_x.push_back(float(k_cube_v[3 * i]) * 0.5f + 0.125f);
        mesh.vertex_y.push_back(float(k_cube_v[3 * i + 1]));
        mesh.vertex_z.push_back(float(k_cube_v[3 * i + 2]) * 3.0f);
    }
    for (std::size_t t = 0; t < 12; ++t) {
        mesh.tri_i0.push_back(Index(k_cube_f[3 * t]));
        mesh.tri_i1.push_back(Index(k_cube_f[3 * t + 1]));
        mesh.tri_i2.push_back(Index(k_cube_f[3 * t + 2]));
    }
    for (bool binary : {true, false}) {
        auto const path = scratch(binary ? "bin.ply" : "ascii.ply");
        CHECK(gwn::gwn_write_ply_mesh(path, mesh, binary).is_ok());
        auto back = gwn::gwn_load_ply_mesh(path);
        CHECK(back.has_value());
        if (back) {
            CHECK(back->vertex_x == mesh.vertex_x && back->vertex_y == mesh.vertex_y && back->vertex_z == mesh.vertex_z);
            CHECK(back->tri_i0 == mesh.tri_i0 && back->tri_i1 == mesh.tri_i1 && back->tri_i2 == mesh.tri_i2);
        }
        std::filesystem::remove(path);
    }
    CHECK(!gwn::gwn_load_ply_mesh(scratch("missing.ply")).has_value());
    gwn::gwn_host_mesh ragged = mesh;
    ragged.tri_i2.pop_back();
    CHECK(gwn::gwn_write_ply_mesh(scratch("ragged.ply"), ragged).error() == gwn::gwn_error::invalid_argument);
}

void eigen_upload_and_scene_files() {
    // a column-major int index matrix and a row-major double vertex matrix give the same geometry
    // as the SoA upload
    gwn::gwn_geometry_object<Real, Index> from_matrix;
    CHECK(gwn::gwn_upload_geometry_from_eigen(from_matrix, fake_matrix<double, true>(8, 3, k_cube_v),
                                              fake_matrix<int, false>(12, 3, k_cube_f))
              .is_ok());
    CHECK(from_matrix.vertex_count() == 8 && from_matrix.triangle_count() == 12);
    auto hx = to_host(from_matrix.accessor().vertex_y);
    auto h2 = to_host(from_matrix.accessor().tri_i2);
    for (std::size_t i = 0; i < 8; ++i)
        CHECK(hx[i] == float(k_cube_v[3 * i + 1]));
    for (std::size_t t = 0; t < 12; ++t)
        CHECK(h2[t] == Index(k_cube_f[3 * t + 2]));

    // PLY -> upload -> build -> moments -> scene file -> load: equal Taylor results
    gwn::gwn_host_mesh mesh;
    auto const ply = scratch("scene_mesh.ply");
    {
        gwn::gwn_host_mesh m;
        for (int k = 0; k < 3; ++k) // three nested cubes
            for (std::size_t i = 0; i < 8; ++i) {
                m.vertex_x.push_back(float(k_cube_v[3 * i]) * (1 + k) + 0.1f * k);
                m.vertex_y.push_back(float(k_cube_v[3 * i + 1]) * (1 + k));
                m.vertex_z.push_back(float(k_cube_v[3 * i + 2]) * (1 + k) - 0.2f * k);
            }
        for (int k = 0; k < 3; ++k)
            for (std::size_t t = 0; t < 12; ++t) {
                m.tri_i0.push_back(Index(k_cube_f[3 * t] + 8 * k));
                m.tri_i1.push_back(Index(k_cube_f[3 * t + 1] + 8 * k));
                m.tri_i2.push_back(Index(k_cube_f[3 * t + 2] + 8 * k));
            }
        CHECK(gwn::gwn_write_ply_mesh(ply, m).is_ok());
    }
    CHECK(gwn::gwn_read_ply_mesh(ply, mesh).is_ok());
    std::filesystem::remove(ply);
    gwn::gwn_geometry_object<Real, Index> geometry;
    CHECK(gwn::gwn_upload_geometry(geometry, mesh).is_ok());
    gwn::gwn_bvh4_object<Real, Index> bvh;
    CHECK(gwn::gwn_build_bvh(geometry, bvh).is_ok());
    gwn::gwn_bvh4_moment_object<1, Real, Index> m1;
    gwn::gwn_bvh4_moment_object<2, Real, Index> m2;
    CHECK(gwn::gwn_refit_bvh_moment<1>(bvh, m1).is_ok());
    CHECK(gwn::gwn_refit_bvh_moment<2>(bvh, m2).is_ok());
    auto const scene = scratch("scene.gwnb");
    CHECK(gwn::gwn_save_scene(scene, geometry, bvh, m1, m2).is_ok());

    gwn::gwn_geometry_object<Real, Index> g2;
    gwn::gwn_bvh4_object<Real, Index> b2;
    gwn::gwn_bvh4_moment_object<0, Real, Index> l0;
    gwn::gwn_bvh4_moment_object<1, Real, Index> l1;
    gwn::gwn_bvh4_moment_object<2, Real, Index> l2;
    CHECK(gwn::gwn_refit_bvh_moment<0>(bvh, l0).is_ok()); // replaced by "not saved" on load
    int orders = 0;
    CHECK(gwn::gwn_load_scene(scene, g2, b2, &l0, &l1, &l2, &orders).is_ok());
    CHECK(orders == 6 && !l0.has_data() && l1.accessor().is_valid_for(b2.accessor()) &&
          l2.accessor().is_valid_for(b2.accessor()));
    CHECK(g2.vertex_count() == 24 && g2.triangle_count() == 36 && b2.accessor().revision != bvh.accessor().revision);
    std::vector<float> qx{0.05f, 1.5f, 2.5f, -3.9f, 7}, qy{0.1f, -0.3f, 2.2f, 0.4f, 1}, qz{-0.2f, 0.7f, -2.1f, 3.3f, 0};
    dbuf dx(qx), dy(qy), dz(qz), a(qx.size()), b(qx.size());
    CHECK(gwn::gwn_compute_winding_number_taylor_batch<2>(bvh, m2, dx.in(), dy.in(), dz.in(), a.out()).is_ok());
    CHECK(gwn::gwn_compute_winding_number_taylor_batch<2>(b2, l2, dx.in(), dy.in(), dz.in(), b.out()).is_ok());
    auto ha = a.host();
    auto hb = b.host();
    CHECK(ha == hb);
    CHECK(std::abs(ha[0] - 3) < 2e-2 && std::abs(ha[1] - 2) < 2e-2 && std::abs(ha[4]) < 2e-2);

    // a damaged file is refused and leaves the targets as they were
    {
        std::FILE *f = std::fopen(scene.string().c_str(), "r+b");
        CHECK(f != nullptr);
        if (f) {
            std::fseek(f, 120, SEEK_SET);
            int const c = std::fgetc(f);
            std::fseek(f, 120, SEEK_SET);
            std::fputc(c ^ 0x10, f);
            std::fclose(f);
        }
    }
    auto const *before = b2.accessor().nodes.data();
    auto st = gwn::gwn_load_scene(scene, g2, b2, nullptr, &l1);
    CHECK(st.error() == gwn::gwn_error::invalid_argument && b2.accessor().nodes.data() == before && l1.has_data());
    std::filesystem::remove(scene);
}

} // namespace

int main(int argc, char **argv) {
    if (argc > 1 && std::strcmp(argv[1], "--compile-only") == 0)
        return 0;
    eigen_bridge_refusals();
    ply_round_trip_on_host();
    if (argc > 1 && std::strcmp(argv[1], "--host-checks") == 0) {
        if (g_failures == 0)
            std::printf("dropin_test: host checks passed\n");
        return g_failures == 0 ? 0 : 1;
    }
    leaf_root_build();
    two_triangle_records_and_refit();
    rejected_options_keep_bvh();
    queries_match_cpu();
    distance_and_ray_on_layers();
    open_cube_boundary_and_antipodal();
    eigen_upload_and_scene_files();
    {
        std::uint64_t const before = gwn::gwn_launch_count();
        leaf_root_build();
        CHECK(gwn::gwn_launch_count() > before);
        std::uint64_t reserved = 0, used = 0;
        CHECK(gwn::gwn_memory_stats(reserved, used).is_ok() && reserved >= used);
        CHECK(gwn::gwn_memory_trim().is_ok());
    }
    if (g_failures == 0)
        std::printf("dropin_test: all checks passed\n");
    return g_failures == 0 ? 0 : 1;
}
