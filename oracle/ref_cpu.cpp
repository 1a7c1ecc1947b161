// ref_cpu.cpp -- extern "C" shim over smallgwn's own CPU reference code (TEST INFRASTRUCTURE).
//
// Compiled by oracle/build.py with g++ into oracle/_ref/libgwnrefcpu.so, from the reference
// project's sources where they lie (never copied): the exact brute force of
// tests/reference_cpu.cuh:22-114 and the vendored SideFX HDK Taylor solid-angle tree
// (tests/reference_hdk/UT_SolidAngle.{h,cpp}, UT_Array.cpp), with the small Eigen and oneTBB
// stand-ins under oracle/shims/ in place of those libraries. bench.py's CPU baseline and reference
// arm time these; tests pin the oracle's C restatement against them.
//
// The HDK glue below follows tests/reference_hdk.cuh:18-89 (positions and triangle points into
// HDK_Sample::UT_SolidAngle, computeSolidAngle per query in a parallel_for, scaled by 1 / 4 pi),
// split into build and query so the tree is built once and queries are timed on their own.
#include "reference_cpu.cuh"
#include "reference_hdk/UT_SolidAngle.h"

#include <tbb/blocked_range.h>
#include <tbb/parallel_for.h>

#include <cstdint>
#include <cstring>
#include <exception>
#include <vector>

namespace {

using Real = float;
using Index = std::uint32_t;

struct hdk_tree {
    std::vector<HDK_Sample::UT_Vector3T<Real>> positions;
    std::vector<int> triangle_points;
    HDK_Sample::UT_SolidAngle<Real, Real> solid_angle;
};

} // namespace

extern "C" {

// Worker threads of the parallel loops (0: all hardware threads). Returns the count in effect.
int refcpu_set_threads(int n) {
    tbb_shim::set_threads(n);
    return tbb_shim::threads();
}

// gwn::tests::reference_winding_number_batch<float> (tests/reference_cpu.cuh:84-114).
int refcpu_exact(const float *x, const float *y, const float *z, uint64_t nv, const uint32_t *i0,
                 const uint32_t *i1, const uint32_t *i2, uint64_t nt, const float *qx, const float *qy,
                 const float *qz, uint64_t nq, float *out) {
    try {
        auto const s = gwn::tests::reference_winding_number_batch<Real, Index>(
            cuda::std::span<Real const>(x, nv), cuda::std::span<Real const>(y, nv),
            cuda::std::span<Real const>(z, nv), cuda::std::span<Index const>(i0, nt),
            cuda::std::span<Index const>(i1, nt), cuda::std::span<Index const>(i2, nt),
            cuda::std::span<Real const>(qx, nq), cuda::std::span<Real const>(qy, nq),
            cuda::std::span<Real const>(qz, nq), cuda::std::span<Real>(out, nq));
        return s.is_ok() ? 0 : 1;
    } catch (...) {
        return 2;
    }
}

// The HDK Taylor tree of a mesh (UT_SolidAngle of `order`, 0..2); nullptr on failure.
void *refcpu_hdk_create(const float *x, const float *y, const float *z, uint64_t nv, const uint32_t *i0,
                        const uint32_t *i1, const uint32_t *i2, uint64_t nt, int order) {
    try {
        if (order < 0 || order > 2 || nv > 0x7fffffffull || nt > 0x7fffffffull)
            return nullptr;
        auto *t = new hdk_tree{};
        t->positions.resize(nv);
        for (uint64_t v = 0; v < nv; ++v) {
            t->positions[v][0] = x[v];
            t->positions[v][1] = y[v];
            t->positions[v][2] = z[v];
        }
        t->triangle_points.resize(3 * nt);
        for (uint64_t i = 0; i < nt; ++i) {
            if (i0[i] >= nv || i1[i] >= nv || i2[i] >= nv) {
                delete t;
                return nullptr;
            }
            t->triangle_points[3 * i + 0] = static_cast<int>(i0[i]);
            t->triangle_points[3 * i + 1] = static_cast<int>(i1[i]);
            t->triangle_points[3 * i + 2] = static_cast<int>(i2[i]);
        }
        t->solid_angle.init(static_cast<int>(nt), t->triangle_points.data(), static_cast<int>(nv),
                            t->positions.data(), order);
        return t;
    } catch (...) {
        return nullptr;
    }
}

// Taylor winding numbers of a query batch at accuracy scale `beta`.
int refcpu_hdk_query(void *tree, const float *qx, const float *qy, const float *qz, uint64_t nq, float beta,
                     float *out) {
    try {
        auto const *t = static_cast<hdk_tree const *>(tree);
        constexpr Real k_pi = Real(3.141592653589793238462643383279502884L);
        Real const inv_4pi = Real(1) / (Real(4) * k_pi);
        tbb::parallel_for(tbb::blocked_range<std::size_t>(0, nq), [&](tbb::blocked_range<std::size_t> const &r) {
            for (std::size_t i = r.begin(); i < r.end(); ++i) {
                HDK_Sample::UT_Vector3T<Real> q{};
                q[0] = qx[i];
                q[1] = qy[i];
                q[2] = qz[i];
                out[i] = t->solid_angle.computeSolidAngle(q, beta) * inv_4pi;
            }
        });
        return 0;
    } catch (...) {
        return 2;
    }
}

void refcpu_hdk_destroy(void *tree) { delete static_cast<hdk_tree *>(tree); }

} // extern "C"
