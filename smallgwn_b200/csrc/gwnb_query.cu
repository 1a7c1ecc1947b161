// Winding-number queries.
//
// Exact batch (replaces gwn_compute_winding_number_exact_batch, gwn_query.cuh:308-346): every CTA
// stages tiles of triangle records in shared memory, each thread evaluates its queries against
// the tile with broadcast shared loads. The solid angle is the Van Oosterom-Strackee formula in
// unnormalised form, tan(Omega/2) = a.(e1 x e2) / (|a||b||c| + (a.b)|c| + (a.c)|b| + (b.c)|a|),
// which equals smallgwn's unit-vector form (detail/gwn_query_geometry_impl.cuh:16-45) and keeps
// its conventions: zero when the query sits on a vertex or the numerator vanishes. Pairs where
// both terms cancel (query by an edge's line) are re-evaluated in FP64 (solid_angle_guarded).
//
// Taylor batch (replaces gwn_compute_winding_number_taylor_batch, gwn_query.cuh:384-445): the
// traversal order, acceptance test and far-field terms follow detail/gwn_query_winding_impl.cuh
// :101-374 (accept a child iff |q-P|^2 > 0, |q-P|^2 > r^2 beta^2 and the expansion is finite;
// otherwise enter internal children, the last directly and the others through the stack, and sum
// leaf triangles exactly). Differences: the batch is Hilbert-ordered internally for coherence, node
// data comes from a per-node query sidecar with 128-bit loads, the stack lives in shared memory,
// and stack overflow writes NaN and raises a device error bit instead of trapping.
#include "gwnb_field.cuh"

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

namespace gwnb {
namespace {

using namespace field;

// Running sums of many terms of mixed size (up to millions of solid angles per query in the exact
// batch, most of them below an ulp of a running sum near 4 pi). With Compensated the sum is kept in
// FP64: the same two registers as a Kahan/Neumaier pair, one DADD per term instead of six FP32
// operations, and no order dependence -- a float Neumaier sum of the 8.4M-triangle sphere still
// loses up to 3e-5 because its correction term itself grows to ~0.15.
template <bool Compensated> struct accum {
    float s = 0.0f;
    __device__ __forceinline__ void add(float x) { s += x; }
    __device__ __forceinline__ float value() const { return s; }
};
template <> struct accum<true> {
    double s = 0.0;
    __device__ __forceinline__ void add(float x) { s += static_cast<double>(x); }
    __device__ __forceinline__ float value() const { return static_cast<float>(s); }
};

// ---- exact batch --------------------------------------------------------------------------------

constexpr int k_exact_block = 256;
constexpr int k_exact_tile = 256;
constexpr int k_exact_q = 2; // queries per thread

// Block (x, y) takes queries [x * 512, x * 512 + 512) against the y-th of gridDim.y contiguous
// ranges of tiles (every range a whole number of tiles). With one range the result is written to
// `out`; with several, each range's FP64 partial sum goes to partial[y * nq + i] and k_exact_finish
// adds the ranges in order (small query batches split the triangles to fill the GPU).
__global__ void __launch_bounds__(k_exact_block, 3)
    k_exact(triangle const *__restrict__ tris, std::uint64_t nt, float const *__restrict__ qx,
            float const *__restrict__ qy, float const *__restrict__ qz, float *__restrict__ out,
            std::uint64_t nq, double *__restrict__ partial) {
    __shared__ float4 s_tri[k_exact_tile][3];
    std::uint64_t const base = static_cast<std::uint64_t>(blockIdx.x) * (k_exact_block * k_exact_q);
    std::uint64_t const tiles = (nt + k_exact_tile - 1) / k_exact_tile;
    std::uint64_t const per = (tiles + gridDim.y - 1) / gridDim.y;
    std::uint64_t const t_begin = static_cast<std::uint64_t>(blockIdx.y) * per * k_exact_tile;
    std::uint64_t const t_end = std::min<std::uint64_t>(t_begin + per * k_exact_tile, nt);
    float px[k_exact_q], py[k_exact_q], pz[k_exact_q];
    accum<true> acc[k_exact_q];
#pragma unroll
    for (int k = 0; k < k_exact_q; ++k) {
        std::uint64_t const i = base + threadIdx.x + static_cast<std::uint64_t>(k) * k_exact_block;
        bool const v = i < nq;
        px[k] = v ? qx[i] : 0.0f;
        py[k] = v ? qy[i] : 0.0f;
        pz[k] = v ? qz[i] : 0.0f;
    }
    for (std::uint64_t t0 = t_begin; t0 < t_end; t0 += k_exact_tile) {
        __syncthreads();
        std::uint64_t const t = t0 + threadIdx.x;
        if (threadIdx.x < k_exact_tile) {
            if (t < t_end) {
                triangle const r = tris[t];
                float const nx = r.e1_y * r.e2_z - r.e1_z * r.e2_y;
                float const ny = r.e1_z * r.e2_x - r.e1_x * r.e2_z;
                float const nz = r.e1_x * r.e2_y - r.e1_y * r.e2_x;
                s_tri[threadIdx.x][0] = make_float4(r.v0_x, r.v0_y, r.v0_z, r.e1_x);
                s_tri[threadIdx.x][1] = make_float4(r.e1_y, r.e1_z, r.e2_x, r.e2_y);
                s_tri[threadIdx.x][2] = make_float4(r.e2_z, nx, ny, nz);
            } else {
                // padding triangle at infinity-free origin with zero edges contributes 0
                s_tri[threadIdx.x][0] = make_float4(0, 0, 0, 0);
                s_tri[threadIdx.x][1] = make_float4(0, 0, 0, 0);
                s_tri[threadIdx.x][2] = make_float4(0, 0, 0, 0);
            }
        }
        __syncthreads();
        std::uint64_t const rem = t_end - t0;
        int const cnt = rem < static_cast<std::uint64_t>(k_exact_tile) ? static_cast<int>(rem) : k_exact_tile;
#pragma unroll 2
        for (int j = 0; j < cnt; ++j) {
            float4 const A = s_tri[j][0];
            float4 const B = s_tri[j][1];
            float4 const C = s_tri[j][2];
#pragma unroll
            for (int k = 0; k < k_exact_q; ++k)
                acc[k].add(solid_angle_guarded(A.x - px[k], A.y - py[k], A.z - pz[k], A.w, B.x, B.y, B.z,
                                               B.w, C.x, C.y, C.z, C.w));
        }
    }
#pragma unroll
    for (int k = 0; k < k_exact_q; ++k) {
        std::uint64_t const i = base + threadIdx.x + static_cast<std::uint64_t>(k) * k_exact_block;
        if (i >= nq)
            continue;
        if (partial == nullptr)
            out[i] = acc[k].value() / (4.0f * k_pi_f);
        else
            partial[static_cast<std::uint64_t>(blockIdx.y) * nq + i] = acc[k].s;
    }
}

__global__ void __launch_bounds__(256)
    k_exact_finish(double const *__restrict__ partial, unsigned ranges, float *__restrict__ out, std::uint64_t nq) {
    std::uint64_t const i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= nq)
        return;
    double s = 0.0;
    for (unsigned r = 0; r < ranges; ++r)
        s += partial[static_cast<std::uint64_t>(r) * nq + i];
    out[i] = static_cast<float>(s) / (4.0f * k_pi_f);
}

// ---- FP64 exact over the float geometry ---------------------------------------------------------

constexpr int k_f64_tile = 128;

__global__ void __launch_bounds__(k_exact_block)
    k_exact_f64(gwnb_geometry_f32 g, float const *__restrict__ qx, float const *__restrict__ qy,
                float const *__restrict__ qz, double *__restrict__ out, std::uint64_t nq) {
    __shared__ double s_v[k_f64_tile][9];
    std::uint64_t const i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    double const px = i < nq ? qx[i] : 0.0, py = i < nq ? qy[i] : 0.0, pz = i < nq ? qz[i] : 0.0;
    double acc = 0.0;
    std::uint64_t const nt = g.triangle_count, nv = g.vertex_count;
    for (std::uint64_t t0 = 0; t0 < nt; t0 += k_f64_tile) {
        __syncthreads();
        if (threadIdx.x < k_f64_tile) {
            std::uint64_t const t = t0 + threadIdx.x;
            bool ok = t < nt;
            std::uint32_t a = 0, b = 0, c = 0;
            if (ok) {
                a = g.tri_i0[t];
                b = g.tri_i1[t];
                c = g.tri_i2[t];
                ok = a < nv && b < nv && c < nv;
            }
            if (ok) {
                s_v[threadIdx.x][0] = g.vertex_x[a];
                s_v[threadIdx.x][1] = g.vertex_y[a];
                s_v[threadIdx.x][2] = g.vertex_z[a];
                s_v[threadIdx.x][3] = g.vertex_x[b];
                s_v[threadIdx.x][4] = g.vertex_y[b];
                s_v[threadIdx.x][5] = g.vertex_z[b];
                s_v[threadIdx.x][6] = g.vertex_x[c];
                s_v[threadIdx.x][7] = g.vertex_y[c];
                s_v[threadIdx.x][8] = g.vertex_z[c];
            } else {
                for (int k = 0; k < 9; ++k)
                    s_v[threadIdx.x][k] = 0.0; // degenerate point triangle contributes 0
            }
        }
        __syncthreads();
        std::uint64_t const rem = nt - t0;
        int const cnt = rem < static_cast<std::uint64_t>(k_f64_tile) ? static_cast<int>(rem) : k_f64_tile;
        for (int j = 0; j < cnt; ++j) {
            double const ax = s_v[j][0] - px, ay = s_v[j][1] - py, az = s_v[j][2] - pz;
            double const bx = s_v[j][3] - px, by = s_v[j][4] - py, bz = s_v[j][5] - pz;
            double const cx = s_v[j][6] - px, cy = s_v[j][7] - py, cz = s_v[j][8] - pz;
            double const la = sqrt(ax * ax + ay * ay + az * az);
            double const lb = sqrt(bx * bx + by * by + bz * bz);
            double const lc = sqrt(cx * cx + cy * cy + cz * cz);
            if (la == 0.0 || lb == 0.0 || lc == 0.0)
                continue;
            double const num = ax * (by * cz - bz * cy) + ay * (bz * cx - bx * cz) + az * (bx * cy - by * cx);
            if (num == 0.0)
                continue;
            double const den = la * lb * lc + (ax * bx + ay * by + az * bz) * lc + (ax * cx + ay * cy + az * cz) * lb +
                               (bx * cx + by * cy + bz * cz) * la;
            acc += 2.0 * atan2(num, den);
        }
    }
    if (i < nq)
        out[i] = acc / (4.0 * 3.141592653589793238462643383279502884);
}

// ---- query ordering -----------------------------------------------------------------------------

__global__ void __launch_bounds__(256)
    k_query_codes(float const *__restrict__ qx, float const *__restrict__ qy,
                  float const *__restrict__ qz, std::uint64_t n, aabb const *__restrict__ root,
                  std::uint32_t *__restrict__ codes) {
    std::uint64_t const i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    codes[i] = hilbert_code30(*root, qx[i], qy[i], qz[i]);
}

// ---- Taylor traversal ---------------------------------------------------------------------------

struct taylor_params {
    float4 const *qnodes;
    std::uint32_t const *qcounts;
    triangle48 const *tri48;
    std::uint64_t primitive_count;
    std::uint64_t node_count;
    std::uint64_t root_ref; // packed reference of the root
    float const *qx;
    float const *qy;
    float const *qz;
    std::uint32_t const *order; // sorted position -> query index (nullptr: identity)
    int gathered;               // 1: qx/qy/qz are already in sorted order (read at the sorted position)
    float *out;
    float *grad_x;
    float *grad_y;
    float *grad_z;
    std::uint32_t *stat_nodes;
    std::uint32_t *stat_far;
    std::uint32_t *stat_near;
    std::uint32_t *stat_union;      // warp form: nodes the query's warp walked (nullptr: not recorded)
    std::uint32_t *stat_union_near; // warp form: leaf triangles the query's warp evaluated
    // Sampled walk (0: every ordered position is walked by this launch), on units of 32 consecutive
    // warps (1,024 ordered positions): local unit u walks the ordered positions of unit
    // u * sample_stride, and local warp w writes {nodes walked, triangles walked, largest per-query
    // nodes, largest per-query triangles} to warp_stats[4 w ...].
    std::uint64_t sample_stride;
    std::uint32_t *warp_stats;
    // per-thread walk: entries of this thread's shared-memory stack column when below the kernel's
    // Cap (the BVH's internal stack bound, so that more blocks fit an SM); 0: Cap
    int thread_stack_cap;
    std::uint64_t n;
    float beta2;
    float fp64_threshold;
    unsigned long long *fp64_count;
    unsigned int *status;
};

// One query of the per-thread traversal: sorted position idx of the batch described by p, with
// s_stack pointing at this thread's column of a [Cap][blockDim.x] shared-memory stack.
template <int Order, int Cap, int Mode, bool Grad, bool Stats>
__device__ __forceinline__ void taylor_thread_item(taylor_params const &p, std::uint64_t idx,
                                                   std::uint32_t *s_stack) {
    constexpr int Q = qnode_traits<Order>::k_f4_per_child;
    if (idx >= p.n)
        return;
    std::uint32_t const qi = p.order != nullptr ? p.order[idx] : static_cast<std::uint32_t>(idx);
    std::uint64_t const li = p.gathered ? idx : qi;
    float const qx = p.qx[li], qy = p.qy[li], qz = p.qz[li];
    accum<Mode == GWNB_NEAR_COMPENSATED> omega;
    float gx = 0.0f, gy = 0.0f, gz = 0.0f;
    std::uint32_t st_nodes = 0, st_far = 0, st_near = 0;
    unsigned const stride = blockDim.x;
    std::uint32_t *const stack = s_stack; // this thread's column; entries are blockDim.x apart
    int const cap = p.thread_stack_cap > 0 && p.thread_stack_cap < Cap ? p.thread_stack_cap : Cap;
    int sp = 0;
    bool overflow = false;

    auto leaf = [&](std::uint32_t first, std::uint32_t cnt) {
        for (std::uint32_t k = 0; k < cnt; ++k) {
            std::uint64_t const t = static_cast<std::uint64_t>(first) + k;
            if (t >= p.primitive_count)
                break;
            float4 const A = __ldg(&p.tri48[t].a);
            float4 const B = __ldg(&p.tri48[t].b);
            float4 const C = __ldg(&p.tri48[t].c);
            float const ax = A.x - qx, ay = A.y - qy, az = A.z - qz;
            if constexpr (Mode == GWNB_NEAR_COMPENSATED)
                omega.add(solid_angle_comp(ax, ay, az, A.w, B.x, B.y, B.z, B.w, C.x, C.y, C.z, C.w,
                                           p.fp64_threshold, p.fp64_count));
            else
                omega.add(solid_angle_plain(ax, ay, az, A.w, B.x, B.y, B.z, B.w, C.x, C.y, C.z, C.w));
            if constexpr (Grad) {
                float3 const g = solid_angle_grad(ax, ay, az, A.w, B.x, B.y, B.z, B.w, C.x);
                gx += g.x;
                gy += g.y;
                gz += g.z;
            }
            if constexpr (Stats)
                ++st_near;
        }
    };

    if (ref_leaf(p.root_ref)) {
        leaf(static_cast<std::uint32_t>(ref_offset(p.root_ref)), ref_count(p.root_ref));
    } else {
        std::uint32_t node = static_cast<std::uint32_t>(ref_offset(p.root_ref));
        for (;;) {
            if (node >= p.node_count)
                break;
            if constexpr (Stats)
                ++st_nodes;
            float4 const *nd = p.qnodes + static_cast<std::uint64_t>(node) * (4 * Q);
            std::uint32_t next = k_invalid_u32;
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                float4 const a = __ldg(nd + s * Q);
                if (a.w < 0.0f)
                    continue;
                float4 const b = __ldg(nd + s * Q + 1);
                float const rx = qx - a.x, ry = qy - a.y, rz = qz - a.z;
                float const q2 = accept_dist2(rx, ry, rz);
                bool descend = !far_accepted(q2, a.w, p.beta2);
                if (!descend) {
                    float g0 = 0.0f, g1 = 0.0f, g2 = 0.0f;
                    float const w = far_field<Order, Grad>(rx, ry, rz, q2, b, nd + s * Q + 2, g0, g1, g2);
                    if (isfinite(w)) {
                        omega.add(w);
                        if constexpr (Grad) {
                            gx += g0;
                            gy += g1;
                            gz += g2;
                        }
                        if constexpr (Stats)
                            ++st_far;
                        continue;
                    }
                }
                std::uint32_t const ref = __float_as_uint(b.w);
                if ((ref & k_qref_leaf) == 0u) {
                    if (next != k_invalid_u32) {
                        if (sp >= cap) {
                            overflow = true;
                            break;
                        }
                        stack[static_cast<unsigned>(sp) * stride] = next;
                        ++sp;
                    }
                    next = ref;
                } else {
                    std::uint32_t const cnt = (ref & k_qref_multi) ? p.qcounts[static_cast<std::uint64_t>(node) * 4 + s] : 1u;
                    leaf(ref & k_qref_index_mask, cnt);
                }
            }
            if (overflow)
                break;
            if (next != k_invalid_u32) {
                node = next;
                continue;
            }
            if (sp == 0)
                break;
            --sp;
            node = stack[static_cast<unsigned>(sp) * stride];
        }
    }
    float const inv4pi = 1.0f / (4.0f * k_pi_f);
    if (overflow) {
        atomicOr(p.status, k_err_stack_overflow);
        float const nan = __int_as_float(0x7fc00000);
        if (p.out != nullptr)
            p.out[qi] = nan;
        if constexpr (Grad) {
            p.grad_x[qi] = nan;
            p.grad_y[qi] = nan;
            p.grad_z[qi] = nan;
        }
        return;
    }
    if (p.out != nullptr)
        p.out[qi] = omega.value() / (4.0f * k_pi_f);
    if constexpr (Grad) {
        p.grad_x[qi] = gx * inv4pi;
        p.grad_y[qi] = gy * inv4pi;
        p.grad_z[qi] = gz * inv4pi;
    }
    if constexpr (Stats) {
        p.stat_nodes[qi] = st_nodes;
        p.stat_far[qi] = st_far;
        p.stat_near[qi] = st_near;
    }
}

template <int Order, int Cap, int Mode, bool Grad, bool Stats>
__global__ void __launch_bounds__(256) k_taylor(taylor_params p) {
    extern __shared__ std::uint32_t s_stack[]; // [Cap][blockDim.x]
    taylor_thread_item<Order, Cap, Mode, Grad, Stats>(
        p, static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x, s_stack + threadIdx.x);
}

// Warp-cooperative traversal: the 32 lanes of a warp (32 Hilbert-adjacent queries) walk one
// depth-first traversal together. Every stack entry carries the mask of lanes that still need the
// subtree; a lane leaves a subtree as soon as it accepts the child's far field. Node records are
// loaded with warp-uniform addresses and the stack lives in the lanes' registers (lane k holds
// entries k and k + 32), so control flow stays uniform. For every lane the nodes it needs are
// visited in the same order as in an independent depth-first traversal (children in decreasing
// slot order, contributions added in slot order), so the per-lane sums equal those of k_taylor.
// Occupancy: the plain form fits 48 registers (5 resident blocks of 256); the compensated near
// field would take ~70, so it is bounded to 4 blocks (64 registers) and the rarely taken FP64 branch
// absorbs any spilling; the gradient and statistics forms also take 4, and the compensated gradient
// 3 (85 registers).
template <int Mode, bool Grad, bool Stats> struct taylor_warp_occupancy {
    static constexpr bool comp = Mode == GWNB_NEAR_COMPENSATED;
    static constexpr int value = (comp && Grad) ? 3 : ((comp || Grad || Stats) ? 4 : 5);
};

// Block shape of the single-BVH warp kernel. The block size changes no result (every warp walks
// its own 32 queries), so the launch does not take the caller's: the compensated value form runs
// 8 blocks of 128 (the same 32 warps and 64 registers as 4 of 256, but a block's warp slots come
// free when its 4 warps are done rather than 8; 1 % less kernel time on the 10M-query workload),
// the other forms blocks of 256.
template <int Mode, bool Grad, bool Stats> struct taylor_warp_shape {
    static constexpr bool small = Mode == GWNB_NEAR_COMPENSATED && !Grad && !Stats;
    static constexpr int block = small ? 128 : 256;
    static constexpr int blocks = small ? 8 : taylor_warp_occupancy<Mode, Grad, Stats>::value;
};

// One warp of the warp-cooperative traversal: lane k takes sorted position idx (idx - lane is the
// warp's first position). Every lane of the warp must call it with the same p.
template <int Order, int Cap, int Mode, bool Grad, bool Stats>
__device__ __forceinline__ void taylor_warp_item(taylor_params const &p, std::uint64_t idx) {
    static_assert(Cap <= 64, "warp stack holds at most 64 entries");
    constexpr int Q = qnode_traits<Order>::k_f4_per_child;
    unsigned const lane = threadIdx.x & 31u;
    bool const valid = idx < p.n;
    unsigned const full = __ballot_sync(0xffffffffu, valid);
    if (full == 0u)
        return;
    // ordered position: idx itself, or the sampled unit's positions in a sampled launch (units of 32
    // consecutive warps, so that a sampled unit's warps share node records in L1 as the batch's do)
    std::uint64_t const pos = p.sample_stride != 0 ? (idx >> 10) * p.sample_stride * 1024 + (idx & 1023u) : idx;
    std::uint32_t const qi = valid ? (p.order != nullptr ? p.order[pos] : static_cast<std::uint32_t>(pos)) : 0u;
    std::uint64_t const li = p.gathered ? pos : qi;
    float const qx = valid ? p.qx[li] : 0.0f;
    float const qy = valid ? p.qy[li] : 0.0f;
    float const qz = valid ? p.qz[li] : 0.0f;
    accum<Mode == GWNB_NEAR_COMPENSATED> omega;
    float gx = 0.0f, gy = 0.0f, gz = 0.0f;
    std::uint32_t st_nodes = 0, st_far = 0, st_near = 0;
    std::uint32_t st_union = 0, st_union_near = 0; // the warp's own work (the same in every lane)

    auto leaf = [&](std::uint32_t first, std::uint32_t cnt) {
        for (std::uint32_t k = 0; k < cnt; ++k) {
            std::uint64_t const t = static_cast<std::uint64_t>(first) + k;
            if (t >= p.primitive_count)
                break;
            float4 const A = __ldg(&p.tri48[t].a);
            float4 const B = __ldg(&p.tri48[t].b);
            float4 const C = __ldg(&p.tri48[t].c);
            float const ax = A.x - qx, ay = A.y - qy, az = A.z - qz;
            if constexpr (Mode == GWNB_NEAR_COMPENSATED)
                omega.add(solid_angle_comp(ax, ay, az, A.w, B.x, B.y, B.z, B.w, C.x, C.y, C.z, C.w,
                                           p.fp64_threshold, p.fp64_count));
            else
                omega.add(solid_angle_plain(ax, ay, az, A.w, B.x, B.y, B.z, B.w, C.x, C.y, C.z, C.w));
            if constexpr (Grad) {
                float3 const g = solid_angle_grad(ax, ay, az, A.w, B.x, B.y, B.z, B.w, C.x);
                gx += g.x;
                gy += g.y;
                gz += g.z;
            }
            if constexpr (Stats)
                ++st_near;
        }
    };

    bool overflow = false;
    if (ref_leaf(p.root_ref)) {
        if (valid)
            leaf(static_cast<std::uint32_t>(ref_offset(p.root_ref)), ref_count(p.root_ref));
    } else {
        std::uint32_t node = static_cast<std::uint32_t>(ref_offset(p.root_ref));
        unsigned mask = full;
        // distributed stack: entry e lives in lane e & 31, bank e >> 5
        std::uint32_t st_node0 = 0, st_node1 = 0;
        unsigned st_mask0 = 0, st_mask1 = 0;
        int sp = 0;
        for (;;) {
            if (node >= p.node_count)
                break;
            bool const active = ((mask >> lane) & 1u) != 0u;
            if constexpr (Stats) {
                st_nodes += active ? 1u : 0u;
                ++st_union;
            }
            float4 const *nd = p.qnodes + static_cast<std::uint64_t>(node) * (4 * Q);
            std::uint32_t next = k_invalid_u32;
            unsigned next_mask = 0u;
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                float4 const a = __ldg(nd + s * Q);
                if (a.w < 0.0f)
                    continue;
                float4 const b = __ldg(nd + s * Q + 1);
                bool desc = false;
                if (active) {
                    float const rx = qx - a.x, ry = qy - a.y, rz = qz - a.z;
                    float const q2 = accept_dist2(rx, ry, rz);
                    desc = !far_accepted(q2, a.w, p.beta2);
                    if (!desc) {
                        float g0 = 0.0f, g1 = 0.0f, g2 = 0.0f;
                        float const w = far_field<Order, Grad>(rx, ry, rz, q2, b, nd + s * Q + 2, g0, g1, g2);
                        if (isfinite(w)) {
                            omega.add(w);
                            if constexpr (Grad) {
                                gx += g0;
                                gy += g1;
                                gz += g2;
                            }
                            if constexpr (Stats)
                                ++st_far;
                        } else {
                            desc = true;
                        }
                    }
                }
                unsigned const dmask = __ballot_sync(0xffffffffu, desc);
                if (dmask == 0u)
                    continue;
                std::uint32_t const ref = __float_as_uint(b.w);
                if ((ref & k_qref_leaf) == 0u) {
                    if (next != k_invalid_u32) {
                        if (sp >= Cap) {
                            overflow = true;
                            break;
                        }
                        if (static_cast<unsigned>(sp & 31) == lane) {
                            if (sp < 32) {
                                st_node0 = next;
                                st_mask0 = next_mask;
                            } else {
                                st_node1 = next;
                                st_mask1 = next_mask;
                            }
                        }
                        ++sp;
                    }
                    next = ref;
                    next_mask = dmask;
                } else {
                    if constexpr (Stats) // the warp runs the leaf loop for its descending lanes
                        st_union_near +=
                            (ref & k_qref_multi) ? p.qcounts[static_cast<std::uint64_t>(node) * 4 + s] : 1u;
                    if (desc) {
                        std::uint32_t const cnt =
                            (ref & k_qref_multi) ? p.qcounts[static_cast<std::uint64_t>(node) * 4 + s] : 1u;
                        leaf(ref & k_qref_index_mask, cnt);
                    }
                }
            }
            if (overflow)
                break;
            if (next != k_invalid_u32) {
                node = next;
                mask = next_mask;
                continue;
            }
            if (sp == 0)
                break;
            --sp;
            int const src = sp & 31;
            if (sp < 32) {
                node = __shfl_sync(0xffffffffu, st_node0, src);
                mask = __shfl_sync(0xffffffffu, st_mask0, src);
            } else {
                node = __shfl_sync(0xffffffffu, st_node1, src);
                mask = __shfl_sync(0xffffffffu, st_mask1, src);
            }
        }
    }
    if constexpr (Stats) {
        if (p.warp_stats != nullptr) {
            std::uint32_t const mn = __reduce_max_sync(0xffffffffu, valid ? st_nodes : 0u);
            std::uint32_t const mt = __reduce_max_sync(0xffffffffu, valid ? st_near : 0u);
            if (lane == 0) {
                std::uint32_t *const w = p.warp_stats + 4 * (idx >> 5);
                w[0] = st_union;
                w[1] = st_union_near;
                w[2] = mn;
                w[3] = mt;
            }
        }
    }
    if (!valid)
        return;
    float const inv4pi = 1.0f / (4.0f * k_pi_f);
    if (overflow) {
        atomicOr(p.status, k_err_stack_overflow);
        float const nan = __int_as_float(0x7fc00000);
        if (p.out != nullptr)
            p.out[qi] = nan;
        if constexpr (Grad) {
            p.grad_x[qi] = nan;
            p.grad_y[qi] = nan;
            p.grad_z[qi] = nan;
        }
        return;
    }
    if (p.out != nullptr)
        p.out[qi] = omega.value() / (4.0f * k_pi_f);
    if constexpr (Grad) {
        p.grad_x[qi] = gx * inv4pi;
        p.grad_y[qi] = gy * inv4pi;
        p.grad_z[qi] = gz * inv4pi;
    }
    if constexpr (Stats) {
        if (p.stat_nodes != nullptr) {
            p.stat_nodes[qi] = st_nodes;
            p.stat_far[qi] = st_far;
            p.stat_near[qi] = st_near;
        }
        if (p.stat_union != nullptr) {
            p.stat_union[qi] = st_union;
            p.stat_union_near[qi] = st_union_near;
        }
    }
}

template <int Order, int Cap, int Mode, bool Grad, bool Stats>
__global__ void __launch_bounds__((taylor_warp_shape<Mode, Grad, Stats>::block),
                                  (taylor_warp_shape<Mode, Grad, Stats>::blocks))
    k_taylor_warp(taylor_params p) {
    taylor_warp_item<Order, Cap, Mode, Grad, Stats>(p, static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x);
}

// ---- batched traversal (many BVHs, one persistent launch) -----------------------------------------
//
// Mesh m owns warps [warp_begin[m], warp_begin[m + 1]) of a global slot space (its queries padded
// to whole warps, so no warp spans two BVHs). The grid strides over warps; a warp finds its mesh by
// binary search (a warp-uniform result) and runs the single-BVH traversal on its 32 slots.

__device__ __forceinline__ std::uint32_t find_mesh_warp(std::uint64_t const *begin, std::uint32_t mesh_count,
                                                        std::uint64_t w) {
    std::uint32_t lo = 0, hi = mesh_count;
    while (hi - lo > 1) {
        std::uint32_t const mid = (lo + hi) >> 1;
        if (__ldg(begin + mid) <= w)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

template <int Order, int Cap, int Mode>
__global__ void __launch_bounds__(256, (taylor_warp_occupancy<Mode, false, false>::value))
    k_batch_taylor_warp(taylor_params const *__restrict__ meshes, std::uint64_t const *__restrict__ warp_begin,
                        std::uint32_t mesh_count, std::uint64_t warps) {
    std::uint64_t const warps_per_grid = static_cast<std::uint64_t>(gridDim.x) * (blockDim.x >> 5);
    for (std::uint64_t w = static_cast<std::uint64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); w < warps;
         w += warps_per_grid) {
        std::uint32_t const m = find_mesh_warp(warp_begin, mesh_count, w);
        taylor_warp_item<Order, Cap, Mode, false, false>(meshes[m], (w - warp_begin[m]) * 32 + (threadIdx.x & 31u));
    }
}

template <int Order, int Cap, int Mode>
__global__ void __launch_bounds__(256)
    k_batch_taylor_thread(taylor_params const *__restrict__ meshes, std::uint64_t const *__restrict__ warp_begin,
                          std::uint32_t mesh_count, std::uint64_t warps) {
    extern __shared__ std::uint32_t s_stack[]; // [Cap][blockDim.x]
    std::uint64_t const warps_per_grid = static_cast<std::uint64_t>(gridDim.x) * (blockDim.x >> 5);
    for (std::uint64_t w = static_cast<std::uint64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); w < warps;
         w += warps_per_grid) {
        std::uint32_t const m = find_mesh_warp(warp_begin, mesh_count, w);
        taylor_thread_item<Order, Cap, Mode, false, false>(meshes[m], (w - warp_begin[m]) * 32 + (threadIdx.x & 31u),
                                                           s_stack + threadIdx.x);
    }
}

template <int Order, int Cap, int Mode, bool Grad, bool Stats>
int launch_taylor_warp(taylor_params const &p, cudaStream_t s) {
    constexpr int block = taylor_warp_shape<Mode, Grad, Stats>::block;
    unsigned const grid = static_cast<unsigned>((p.n + block - 1) / block);
    note_launch(), k_taylor_warp<Order, Cap, Mode, Grad, Stats><<<grid, block, 0, s>>>(p);
    GWNB_CUDA_TRY(cudaGetLastError());
    return GWNB_OK;
}

// Per-thread walk: each thread's stack column holds `cap` entries (the BVH's internal stack bound,
// at most Cap): a 46-entry bound fits four blocks of 256 per SM where 64-entry columns fit three.
template <int Order, int Cap, int Mode, bool Grad, bool Stats>
int launch_taylor_cap(taylor_params const &p_in, int block, int cap, cudaStream_t s) {
    taylor_params p = p_in;
    p.thread_stack_cap = cap > 0 && cap < Cap ? cap : Cap;
    std::size_t const smem = static_cast<std::size_t>(p.thread_stack_cap) * block * sizeof(std::uint32_t);
    auto kern = k_taylor<Order, Cap, Mode, Grad, Stats>;
    if (smem > 48 * 1024)
        GWNB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           static_cast<int>(smem)));
    unsigned const grid = static_cast<unsigned>((p.n + block - 1) / block);
    note_launch(), kern<<<grid, block, smem, s>>>(p);
    GWNB_CUDA_TRY(cudaGetLastError());
    return GWNB_OK;
}

template <int Order, int Mode, bool Grad, bool Stats>
int launch_taylor_mode(taylor_params const &p, int block, int cap, bool per_thread, cudaStream_t s) {
    if (!per_thread && cap <= 32)
        return launch_taylor_warp<Order, 32, Mode, Grad, Stats>(p, s);
    if (!per_thread && cap <= 64)
        return launch_taylor_warp<Order, 64, Mode, Grad, Stats>(p, s);
    if (cap <= 16)
        return launch_taylor_cap<Order, 16, Mode, Grad, Stats>(p, block, cap, s);
    if (cap <= 32)
        return launch_taylor_cap<Order, 32, Mode, Grad, Stats>(p, block, cap, s);
    if (cap <= 64)
        return launch_taylor_cap<Order, 64, Mode, Grad, Stats>(p, block, cap, s);
    return launch_taylor_cap<Order, 128, Mode, Grad, Stats>(p, block, cap, s);
}

template <int Order, bool Grad, bool Stats>
int launch_taylor_order(taylor_params const &p, int block, int cap, int mode, bool per_thread, cudaStream_t s) {
    if (mode == GWNB_NEAR_COMPENSATED)
        return launch_taylor_mode<Order, GWNB_NEAR_COMPENSATED, Grad, Stats>(p, block, cap, per_thread, s);
    return launch_taylor_mode<Order, GWNB_NEAR_PLAIN, Grad, Stats>(p, block, cap, per_thread, s);
}

} // namespace

int exact_batch(triangle const *tris, std::uint64_t nt, float const *qx, float const *qy,
                float const *qz, float *out, std::uint64_t nq, cudaStream_t s) {
    if (nq == 0)
        return GWNB_OK;
    std::uint64_t const qblocks = (nq + k_exact_block * k_exact_q - 1) / (k_exact_block * k_exact_q);
    // Split the triangles into ranges of at least 4 tiles until ~6 blocks per SM are in flight
    // (3 are resident at 72 registers); one range writes the result directly.
    std::uint64_t const tiles = (nt + k_exact_tile - 1) / k_exact_tile;
    std::uint64_t const want = static_cast<std::uint64_t>(device_sm_count()) * 6;
    std::uint64_t ranges = qblocks >= want ? 1 : (want + qblocks - 1) / qblocks;
    ranges = std::min<std::uint64_t>(ranges, std::max<std::uint64_t>(tiles / 4, 1));
    ranges = std::min<std::uint64_t>(ranges, 64);
    double *partial = nullptr;
    if (ranges > 1)
        GWNB_TRY(alloc(&partial, ranges * nq, s));
    dim3 const grid(static_cast<unsigned>(qblocks), static_cast<unsigned>(ranges));
    note_launch(), k_exact<<<grid, k_exact_block, 0, s>>>(tris, nt, qx, qy, qz, out, nq, partial);
    if (ranges > 1)
        note_launch(), k_exact_finish<<<static_cast<unsigned>((nq + 255) / 256), 256, 0, s>>>(partial, static_cast<unsigned>(ranges),
                                                                             out, nq);
    cudaError_t const e = cudaGetLastError();
    release(partial, s);
    if (e != cudaSuccess)
        return set_cuda_error(e, "exact batch launch");
    return GWNB_OK;
}

int exact_batch_f64(gwnb_geometry_f32 const &g, float const *qx, float const *qy, float const *qz, double *out,
                    std::uint64_t nq, cudaStream_t s) {
    if (nq == 0)
        return GWNB_OK;
    note_launch(), k_exact_f64<<<static_cast<unsigned>((nq + k_exact_block - 1) / k_exact_block), k_exact_block, 0, s>>>(
        g, qx, qy, qz, out, nq);
    GWNB_CUDA_TRY(cudaGetLastError());
    return GWNB_OK;
}

int query_order(aabb const *root_bounds, float const *qx, float const *qy, float const *qz, std::uint64_t n,
                std::uint32_t *order, cudaStream_t s, unsigned int *status) {
    if (n == 0)
        return GWNB_OK;
    std::uint32_t *codes = nullptr, *sorted = nullptr;
    scratch_guard guard(s);
    guard.hold(codes, sorted);
    GWNB_TRY(alloc(&codes, n, s));
    GWNB_TRY(alloc(&sorted, n, s));
    note_launch(), k_query_codes<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(qx, qy, qz, n, root_bounds, codes);
    int const rc = radix_sort_pairs(codes, sorted, nullptr, order, n, 4, 30, s, status);
    release(codes, s);
    release(sorted, s);
    return rc;
}



namespace {
__global__ void __launch_bounds__(256)
    k_gather_queries(std::uint32_t const *__restrict__ order, float const *__restrict__ qx,
                     float const *__restrict__ qy, float const *__restrict__ qz, std::uint64_t n,
                     float *__restrict__ sx, float *__restrict__ sy, float *__restrict__ sz) {
    std::uint64_t const i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    std::uint32_t const j = order[i];
    sx[i] = __ldg(qx + j);
    sy[i] = __ldg(qy + j);
    sz[i] = __ldg(qz + j);
}

taylor_params make_taylor_params(taylor_request const &r) {
    taylor_params p{};
    p.qnodes = r.qnodes;
    p.qcounts = r.qcounts;
    p.tri48 = r.tri48;
    p.primitive_count = r.primitive_count;
    p.node_count = r.node_count;
    p.root_ref = r.root_ref;
    p.qx = r.qx;
    p.qy = r.qy;
    p.qz = r.qz;
    p.out = r.out;
    p.grad_x = r.gx;
    p.grad_y = r.gy;
    p.grad_z = r.gz;
    p.stat_nodes = r.stat_nodes;
    p.stat_far = r.stat_far;
    p.stat_near = r.stat_near;
    p.n = r.n;
    p.beta2 = r.accuracy_scale * r.accuracy_scale;
    p.fp64_threshold = r.fp64_threshold;
    p.fp64_count = r.fp64_count;
    p.status = r.status;
    return p;
}
} // namespace

namespace {

// Which walk suits a batch, from a sample of its own warps walked warp-cooperatively with statistics:
// the per-thread walk pays off where the sampled warps walked at least 1.3 times the nodes of their
// longest single path and that path met at most 8 leaf triangles on average. Every point of the
// measured crossover (per-thread / warp-cooperative kernel time 0.54-0.78 on 1M far-field-heavy
// queries, 1.1-3.0 on surface-heavy or dense batches) outside [0.9, 1.1] falls on the right side of
// the rule; the sample itself is too slow to take before every batch (its few warps run at the
// latency of whole walks), so it stays a diagnostic.
constexpr double k_form_union_ratio = 1.3;
constexpr double k_form_lane_tris = 8.0;

struct form_sample {
    std::uint64_t stride, count; // every stride-th full unit of 32 warps, count of them (0: none)
};

// Every stride-th unit of 32 consecutive ordered warps: one resident wave of units or 1/64 of the
// batch, whichever is more, for batches of at least four waves; up to 64 units below that.
form_sample choose_sample(std::uint64_t n) {
    std::uint64_t const units = n / 1024; // full units
    std::uint64_t const wave = static_cast<std::uint64_t>(device_sm_count()); // units in one resident wave
    if (units == 0)
        return {0, 0};
    std::uint64_t const stride = units < 4 * wave ? std::max<std::uint64_t>(units / 64, 1)
                                                  : std::max<std::uint64_t>(units / std::max(wave, units / 64), 2);
    return {stride, (units + stride - 1) / stride};
}

bool per_thread_wins(double walked, double lane_max, double lane_tris, double count) {
    return walked >= k_form_union_ratio * lane_max && lane_tris <= k_form_lane_tris * count;
}

template <int O> int launch_probe(taylor_params const &p, int cap, int mode, cudaStream_t s) {
    return launch_taylor_order<O, false, true>(p, 256, cap, mode, false, s);
}
int dispatch_probe(int order, taylor_params const &p, int cap, int mode, cudaStream_t s) {
    return order == 0 ? launch_probe<0>(p, cap, mode, s)
                      : (order == 1 ? launch_probe<1>(p, cap, mode, s) : launch_probe<2>(p, cap, mode, s));
}

} // namespace

// Sampled walk statistics of a batch in traversal order `order` (nullptr: the queries are already
// in that order): the sample of choose_sample, walked warp-cooperatively with statistics and no
// outputs; out[0..3] = per sampled warp, nodes walked, triangles walked, longest path nodes, longest
// path triangles; out[4] sampled warps (0 below 1,024 queries); out[5] 1 when the rule above takes
// the per-thread walk. Synchronizes the stream.
int taylor_probe(taylor_request const &r, std::uint32_t const *order, cudaStream_t s, double out[6]) {
    for (int k = 0; k < 6; ++k)
        out[k] = 0.0;
    form_sample const fs = choose_sample(r.n);
    if (fs.count == 0)
        return GWNB_OK;
    std::uint64_t const warps = fs.count * 32;
    std::uint32_t *ws = nullptr;
    GWNB_TRY(alloc(&ws, 4 * warps, s));
    taylor_params p = make_taylor_params(r);
    p.order = order;
    p.gathered = 0;
    p.out = nullptr;
    p.sample_stride = fs.stride;
    p.n = warps * 32;
    p.warp_stats = ws;
    int rc = dispatch_probe(r.order, p, r.stack_capacity, r.near_mode, s);
    std::vector<std::uint32_t> h(4 * warps);
    if (rc == GWNB_OK && (cudaMemcpyAsync(h.data(), ws, h.size() * sizeof(std::uint32_t), cudaMemcpyDeviceToHost, s) !=
                              cudaSuccess ||
                          cudaStreamSynchronize(s) != cudaSuccess))
        rc = set_cuda_error(cudaGetLastError(), "taylor probe read-back");
    release(ws, s);
    if (rc != GWNB_OK)
        return rc;
    double t[4] = {0.0, 0.0, 0.0, 0.0};
    for (std::uint64_t w = 0; w < warps; ++w)
        for (int k = 0; k < 4; ++k)
            t[k] += h[4 * w + k];
    double const c = static_cast<double>(warps);
    for (int k = 0; k < 4; ++k)
        out[k] = t[k] / c;
    out[4] = c;
    out[5] = per_thread_wins(t[0], t[2], t[3], c) ? 1.0 : 0.0;
    return GWNB_OK;
}

// ---- timed choice of the walk (per_thread = 2) -------------------------------------------------------
//
// Both walks give identical results; which one is faster depends on the batch (dense or
// surface-heavy batches favour the warp walk, sparse far-field-heavy ones the per-thread walk). The
// first call of a kind walks warp-cooperatively and the second per thread, each traversal launch
// bracketed by CUDA events; a later call whose two measurements have completed takes the faster
// walk from then on (until then: the warp walk, untimed). A kind is the moment sidecar's address,
// order, precision mode, gradient form, accuracy scale, whether the batch is ordered, the device
// and floor(log2 n). Nothing blocks: the events are polled. Calls under stream capture take the
// decided walk, or the warp walk, and record nothing.
namespace {

struct walk_timing {
    int phase = 0; // 0: nothing timed; 1: warp walk timed; 2: both timed; 3: decided
    bool per_thread = false;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr}; // warp start / end, per-thread start / end
};
constexpr std::size_t k_walk_kinds = 256; // the table is emptied when it holds this many kinds

std::mutex &walk_mutex() {
    static std::mutex m;
    return m;
}
std::map<walk_kind, walk_timing> &walk_table() {
    static auto *t = new std::map<walk_kind, walk_timing>(); // never destroyed: outlives the runtime at exit
    return *t;
}

void destroy_events(walk_timing &t) {
    for (auto &e : t.ev)
        if (e != nullptr) {
            cudaEventDestroy(e);
            e = nullptr;
        }
}

// cudaSuccess when the event has completed, cudaErrorNotReady while it is pending (not left as the
// thread's last error), another code on failure.
cudaError_t poll(cudaEvent_t e) {
    cudaError_t const q = cudaEventQuery(e);
    if (q == cudaErrorNotReady && cudaPeekAtLastError() == cudaErrorNotReady)
        (void)cudaGetLastError();
    return q;
}

} // namespace

walk_plan plan_walk(walk_kind const &k, cudaStream_t s) {
    walk_plan plan;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    bool const capturing = cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone;
    std::lock_guard<std::mutex> lock(walk_mutex());
    auto &table = walk_table();
    auto it = table.find(k);
    if (capturing) {
        plan.per_thread = it != table.end() && it->second.phase == 3 && it->second.per_thread;
        return plan;
    }
    if (it == table.end()) {
        if (table.size() >= k_walk_kinds) {
            for (auto &kv : table)
                destroy_events(kv.second);
            table.clear();
        }
        walk_timing t;
        for (auto &e : t.ev)
            if (cudaEventCreate(&e) != cudaSuccess) {
                (void)cudaGetLastError();
                destroy_events(t);
                return plan; // untimed warp walk
            }
        it = table.emplace(k, t).first;
    }
    walk_timing &t = it->second;
    switch (t.phase) {
    case 0:
        plan.start = t.ev[0];
        plan.stop = t.ev[1];
        t.phase = 1;
        break;
    case 1:
        plan.per_thread = true;
        plan.start = t.ev[2];
        plan.stop = t.ev[3];
        t.phase = 2;
        break;
    case 2: {
        cudaError_t const a = poll(t.ev[1]);
        cudaError_t const b = a == cudaSuccess ? poll(t.ev[3]) : a;
        if (a == cudaErrorNotReady || b == cudaErrorNotReady)
            break; // still pending: warp walk, untimed
        float warp_ms = 0.0f, thread_ms = 0.0f;
        bool const ok = a == cudaSuccess && b == cudaSuccess &&
                        cudaEventElapsedTime(&warp_ms, t.ev[0], t.ev[1]) == cudaSuccess &&
                        cudaEventElapsedTime(&thread_ms, t.ev[2], t.ev[3]) == cudaSuccess;
        if (!ok)
            (void)cudaGetLastError();
        t.per_thread = ok && thread_ms < warp_ms;
        t.phase = 3;
        destroy_events(t);
        plan.per_thread = t.per_thread;
        break;
    }
    default:
        plan.per_thread = t.per_thread;
    }
    return plan;
}

int taylor_batch(taylor_request const &r, cudaStream_t s) {
    if (r.n == 0)
        return GWNB_OK;
    taylor_params p = make_taylor_params(r);
    std::uint32_t *codes = nullptr, *sorted_codes = nullptr, *order = nullptr;
    float *gathered = nullptr;
    scratch_guard guard(s);
    guard.hold(codes, sorted_codes, order, gathered);
    bool const sorted = r.sort_queries != 0 && r.n > 1 && r.root_bounds != nullptr;
    if (sorted) {
        GWNB_NVTX("gwnb::taylor.order");
        GWNB_TRY(alloc(&codes, r.n, s));
        GWNB_TRY(alloc(&sorted_codes, r.n, s));
        GWNB_TRY(alloc(&order, r.n, s));
        note_launch(), k_query_codes<<<static_cast<unsigned>((r.n + 255) / 256), 256, 0, s>>>(r.qx, r.qy, r.qz, r.n,
                                                                            r.root_bounds, codes);
        GWNB_TRY(radix_sort_pairs(codes, sorted_codes, nullptr, order, r.n, 4, 30, s, r.status));
        p.order = order;
        // the queries themselves in traversal order: the traversal then reads them contiguously
        release(sorted_codes, s);
        sorted_codes = nullptr;
        GWNB_TRY(alloc(&gathered, 3 * r.n, s));
        note_launch(), k_gather_queries<<<static_cast<unsigned>((r.n + 255) / 256), 256, 0, s>>>(
            order, r.qx, r.qy, r.qz, r.n, gathered, gathered + r.n, gathered + 2 * r.n);
        p.qx = gathered;
        p.qy = gathered + r.n;
        p.qz = gathered + 2 * r.n;
        p.gathered = 1;
    }
    if (r.probe != nullptr) {
        taylor_request rq = r;
        rq.qx = p.qx;
        rq.qy = p.qy;
        rq.qz = p.qz;
        int const prc = taylor_probe(rq, sorted ? nullptr : p.order, s, r.probe);
        release(codes, s);
        release(order, s);
        release(gathered, s);
        return prc;
    }
    bool const grad = r.gx != nullptr;
    bool const stats = r.stat_nodes != nullptr;
    int rc = GWNB_OK;
    GWNB_NVTX("gwnb::taylor.traverse");
    int const block = query_launch_block(r.block);
    int const cap = r.stack_capacity;
    walk_plan plan;
    plan.per_thread = r.per_thread == 1;
    if (r.per_thread == 2 && !stats) {
        int device = 0;
        (void)cudaGetDevice(&device);
        float const beta = r.accuracy_scale;
        std::uint32_t beta_bits = 0;
        std::memcpy(&beta_bits, &beta, sizeof(beta_bits));
        int size_class = 0;
        for (std::uint64_t v = r.n; v > 1; v >>= 1)
            ++size_class;
        plan = plan_walk(walk_kind{r.qnodes, device, 0, r.order, r.near_mode, grad ? 1 : 0, sorted ? 1 : 0,
                                   size_class, beta_bits},
                         s);
    }
    bool const per_thread = plan.per_thread;
    if (plan.start != nullptr)
        (void)cudaEventRecord(plan.start, s);
#define GWNB_DISPATCH(O)                                                                           \
    if (grad)                                                                                      \
        rc = launch_taylor_order<O, true, false>(p, block, cap, r.near_mode, per_thread, s);       \
    else if (stats)                                                                                \
        rc = launch_taylor_order<O, false, true>(p, block, cap, r.near_mode, per_thread, s);       \
    else                                                                                           \
        rc = launch_taylor_order<O, false, false>(p, block, cap, r.near_mode, per_thread, s);
    if (r.order == 0) {
        GWNB_DISPATCH(0)
    } else if (r.order == 1) {
        GWNB_DISPATCH(1)
    } else {
        GWNB_DISPATCH(2)
    }
#undef GWNB_DISPATCH
    if (plan.stop != nullptr)
        (void)cudaEventRecord(plan.stop, s);
    release(codes, s);
    release(sorted_codes, s);
    release(order, s);
    release(gathered, s);
    return rc;
}

// ---- batched traversal (host) -----------------------------------------------------------------------

int batch_query_prepare(taylor_request const *reqs, std::uint32_t n, batch_query_state *st, cudaStream_t s) {
    std::vector<taylor_params> sorted(n), unsorted(n);
    std::vector<std::uint64_t> wb(n + 1, 0);
    std::uint64_t total = 0;
    int max_bound = 1;
    for (std::uint32_t i = 0; i < n; ++i) {
        total += reqs[i].n;
        wb[i + 1] = wb[i] + (reqs[i].n + 31) / 32;
        max_bound = std::max(max_bound, reqs[i].stack_capacity);
    }
    GWNB_TRY(alloc(&st->orders, std::max<std::uint64_t>(total, 1), s));
    std::uint64_t off = 0;
    for (std::uint32_t i = 0; i < n; ++i) {
        taylor_params p = make_taylor_params(reqs[i]);
        p.thread_stack_cap = max_bound; // the per-thread kernel's stack columns (launch_batch_cap)
        unsorted[i] = p;
        if (reqs[i].n > 1 && reqs[i].root_bounds != nullptr) {
            GWNB_TRY(query_order(reqs[i].root_bounds, reqs[i].qx, reqs[i].qy, reqs[i].qz, reqs[i].n, st->orders + off, s,
                                 reqs[i].status));
            p.order = st->orders + off;
        }
        sorted[i] = p;
        off += reqs[i].n;
    }
    // each buffer joins the state as soon as it exists, so batch_query_release frees it on any
    // failure after this point
    taylor_params *ds = nullptr, *du = nullptr;
    GWNB_TRY(alloc(&ds, n, s));
    st->meshes = ds;
    GWNB_TRY(alloc(&du, n, s));
    st->meshes_unsorted = du;
    GWNB_TRY(alloc(&st->warp_begin, n + 1, s));
    GWNB_CUDA_TRY(cudaMemcpyAsync(ds, sorted.data(), n * sizeof(taylor_params), cudaMemcpyHostToDevice, s));
    GWNB_CUDA_TRY(cudaMemcpyAsync(du, unsorted.data(), n * sizeof(taylor_params), cudaMemcpyHostToDevice, s));
    GWNB_CUDA_TRY(cudaMemcpyAsync(st->warp_begin, wb.data(), (n + 1) * sizeof(std::uint64_t), cudaMemcpyHostToDevice, s));
    GWNB_CUDA_TRY(cudaStreamSynchronize(s)); // the host vectors go out of scope
    st->mesh_count = n;
    st->order = n > 0 ? reqs[0].order : 0;
    st->near_mode = n > 0 ? reqs[0].near_mode : GWNB_NEAR_PLAIN;
    st->warps = wb[n];
    st->max_stack_bound = max_bound;
    return GWNB_OK;
}

namespace {
template <int Order, int Cap, int Mode>
int launch_batch_cap(batch_query_state const &st, batch_query_config const &c, cudaStream_t s) {
    auto const *meshes = static_cast<taylor_params const *>(c.sorted ? st.meshes : st.meshes_unsorted);
    int const block = c.block;
    std::uint64_t const need = (st.warps * 32 + block - 1) / block;
    std::uint64_t const cap = static_cast<std::uint64_t>(device_sm_count()) * std::max(c.grid_scale, 1);
    unsigned const grid = static_cast<unsigned>(std::max<std::uint64_t>(std::min(need, cap), 1));
    if (c.per_thread == 0) {
        note_launch(), k_batch_taylor_warp<Order, Cap, Mode><<<grid, block, 0, s>>>(meshes, st.warp_begin, st.mesh_count, st.warps);
    } else {
        // stack columns of the batch's largest stack bound (every mesh's thread_stack_cap)
        int const column = st.max_stack_bound > 0 && st.max_stack_bound < Cap ? st.max_stack_bound : Cap;
        std::size_t const smem = static_cast<std::size_t>(column) * block * sizeof(std::uint32_t);
        auto kern = k_batch_taylor_thread<Order, Cap, Mode>;
        if (smem > 48 * 1024)
            GWNB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
        note_launch(), kern<<<grid, block, smem, s>>>(meshes, st.warp_begin, st.mesh_count, st.warps);
    }
    GWNB_CUDA_TRY(cudaGetLastError());
    return GWNB_OK;
}

template <int Order, int Mode>
int launch_batch_mode(batch_query_state const &st, batch_query_config const &c, cudaStream_t s) {
    if (st.max_stack_bound <= 32)
        return launch_batch_cap<Order, 32, Mode>(st, c, s);
    return launch_batch_cap<Order, 64, Mode>(st, c, s);
}

template <int Order>
int launch_batch_order(batch_query_state const &st, batch_query_config const &c, cudaStream_t s) {
    if (st.near_mode == GWNB_NEAR_COMPENSATED)
        return launch_batch_mode<Order, GWNB_NEAR_COMPENSATED>(st, c, s);
    return launch_batch_mode<Order, GWNB_NEAR_PLAIN>(st, c, s);
}
} // namespace

int batch_query_launch(batch_query_state const &st, batch_query_config const &c, cudaStream_t s) {
    if (st.warps == 0)
        return GWNB_OK;
    if (c.block < 32 || c.block > 256 || (c.block % 32) != 0)
        return set_error(GWNB_INVALID_ARGUMENT, "Batch query block size must be a multiple of 32 in [32, 256].");
    if (st.max_stack_bound > 64)
        return set_error(GWNB_INVALID_ARGUMENT, "Batched traversal supports stack bounds up to 64.");
    if (st.order == 0)
        return launch_batch_order<0>(st, c, s);
    if (st.order == 1)
        return launch_batch_order<1>(st, c, s);
    return launch_batch_order<2>(st, c, s);
}

void batch_query_release(batch_query_state &st, cudaStream_t s) {
    auto *ds = static_cast<taylor_params *>(st.meshes);
    auto *du = static_cast<taylor_params *>(st.meshes_unsorted);
    release(ds, s);
    release(du, s);
    release(st.warp_begin, s);
    release(st.orders, s);
    st.meshes = nullptr;
    st.meshes_unsorted = nullptr;
}

std::size_t radix_sort_u32_scratch_words(std::uint64_t n, int key_bits);
int radix_sort_pairs_u32_in_scratch(std::uint32_t const *keys_in, std::uint32_t *keys_out,
                                    std::uint32_t const *values_in, std::uint32_t *values_out, std::uint64_t n,
                                    int key_bits, std::uint32_t *keys_tmp, std::uint32_t *vals_tmp,
                                    std::uint32_t *words, cudaStream_t s, unsigned int *status);

// The Taylor batch of taylor_batch() with every temporary in caller-provided scratch (query Hilbert
// codes, sorted codes, the order, the sort's ping-pong buffers and its words); allocates nothing.
int taylor_batch_in_scratch(taylor_request const &r, std::uint32_t *scratch, std::uint64_t capacity,
                            cudaStream_t s) {
    if (r.n == 0)
        return GWNB_OK;
    if (r.n > capacity)
        return set_error(GWNB_INVALID_ARGUMENT, "query batch exceeds the scratch capacity");
    taylor_params p{};
    p.qnodes = r.qnodes;
    p.qcounts = r.qcounts;
    p.tri48 = r.tri48;
    p.primitive_count = r.primitive_count;
    p.node_count = r.node_count;
    p.root_ref = r.root_ref;
    p.qx = r.qx;
    p.qy = r.qy;
    p.qz = r.qz;
    p.out = r.out;
    p.n = r.n;
    p.beta2 = r.accuracy_scale * r.accuracy_scale;
    p.fp64_threshold = r.fp64_threshold;
    p.fp64_count = r.fp64_count;
    p.status = r.status;
    if (r.sort_queries != 0 && r.n > 1 && r.root_bounds != nullptr) {
        // five regions of `capacity` words each, then the sort's words
        std::uint32_t *codes = scratch;
        std::uint32_t *sorted_codes = scratch + capacity;
        std::uint32_t *order = scratch + 2 * capacity;
        std::uint32_t *keys_tmp = scratch + 3 * capacity;
        std::uint32_t *vals_tmp = scratch + 4 * capacity;
        std::uint32_t *words = scratch + 5 * capacity;
        note_launch(), k_query_codes<<<static_cast<unsigned>((r.n + 255) / 256), 256, 0, s>>>(r.qx, r.qy, r.qz, r.n,
                                                                            r.root_bounds, codes);
        GWNB_TRY(radix_sort_pairs_u32_in_scratch(codes, sorted_codes, nullptr, order, r.n, 30, keys_tmp, vals_tmp,
                                                 words, s, r.status));
        p.order = order;
    }
    int const block = query_launch_block(r.block);
    bool const per_thread = r.per_thread != 0;
    if (r.order == 0)
        return launch_taylor_order<0, false, false>(p, block, r.stack_capacity, r.near_mode, per_thread, s);
    if (r.order == 1)
        return launch_taylor_order<1, false, false>(p, block, r.stack_capacity, r.near_mode, per_thread, s);
    return launch_taylor_order<2, false, false>(p, block, r.stack_capacity, r.near_mode, per_thread, s);
}

} // namespace gwnb
